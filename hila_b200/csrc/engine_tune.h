// Decision logic of the engine's launch-shape tuner (host only, no CUDA): which
// candidate shape a chunk runs, what a timed chunk counts for, and when a work class
// is decided.  The engine (engine.cpp) times the chunks; this file only keeps score.
//
// The candidates round every product and sum alike (the packed two-solve hop and the
// one-solve-per-thread hop, each with the dynamic or the fixed tile order), so a
// solve's bits do not depend on the choice.  A work class is the bit length of the
// sum over the running Wilson solves of their lattice's 128-site tiles.
#pragma once

namespace hw {

struct TuneShape {
    int variant;  // EngGrid::variant
    int dyn;      // EngTables::dyn
};

constexpr int kTuneMaxShapes = 4;
constexpr int kTuneSamples = 2;     // counted chunks per candidate
constexpr int kTuneMaxIters = 16;   // iterations of a chunk with events
constexpr int kTuneMinClass = 10;   // smaller batches (< 512 tile-solves, about one wave of
                                    // blocks) run the default shape untimed
constexpr int kTuneAttempts = 4;    // timed chunks per candidate before deciding on what was seen

struct TuneEntry {
    double ms[kTuneMaxShapes] = {};  // lowest median per-iteration time counted
    int samples[kTuneMaxShapes] = {};
    int attempts = 0;  // timed chunks, counted or not
    int next = 0;      // candidate of the next timed chunk
    int chosen = -1;   // index of the fastest, once decided
};

// bit length of the tile-solves of the running Wilson solves
inline int tune_work_class(unsigned long long units) {
    int bits = 0;
    while (units) {
        bits++;
        units >>= 1;
    }
    return bits;
}

// the candidate a chunk of this entry runs; *timed: the chunk is to be timed
inline int tune_pick(const TuneEntry &e, bool *timed) {
    *timed = e.chosen < 0;
    return e.chosen >= 0 ? e.chosen : e.next;
}

// Keep the fastest candidate with a sample (every one with kTuneSamples when `complete`).
inline void tune_decide(TuneEntry &e, int nshapes, bool complete) {
    int best = -1;
    for (int c = 0; c < nshapes; c++) {
        if (complete && e.samples[c] < kTuneSamples) return;
        if (e.samples[c] > 0 && (best < 0 || e.ms[c] < e.ms[best])) best = c;
    }
    e.chosen = best < 0 ? 0 : best;
}

// One timed chunk of candidate `shape`.  counted: every solve ran all its iterations (none
// finished inside the chunk), and ms is the median device time per iteration of the phases
// the shape changes.  An uncounted chunk leaves the next chunk on the same candidate.
// After kTuneAttempts timed chunks per candidate the entry decides on the samples it has
// (a stream whose solves keep finishing inside chunks gives few countable ones).
inline void tune_record(TuneEntry &e, int shape, int nshapes, bool counted, double ms) {
    if (e.chosen >= 0 || shape < 0 || shape >= nshapes) return;
    e.attempts++;
    if (counted) {
        if (e.samples[shape] == 0 || ms < e.ms[shape]) e.ms[shape] = ms;
        e.samples[shape]++;
        e.next = (shape + 1) % nshapes;
        tune_decide(e, nshapes, true);
    }
    if (e.chosen < 0 && e.attempts >= kTuneAttempts * nshapes) tune_decide(e, nshapes, false);
}

}  // namespace hw
