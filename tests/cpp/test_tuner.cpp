// Decision logic of the engine's launch-shape tuner (hila_b200/csrc/engine_tune.h),
// driven with made-up chunk timings: no GPU involved.
#include <cstdio>
#include <cstdlib>

#include "engine_tune.h"

using namespace hw;

static int failures = 0;
#define CHECK(c)                                                    \
    do {                                                            \
        if (!(c)) {                                                 \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #c); \
            failures++;                                             \
        }                                                           \
    } while (0)

int main() {
    // work classes: bit length of the tile-solves
    CHECK(tune_work_class(0) == 0);
    CHECK(tune_work_class(1) == 1);
    CHECK(tune_work_class(511) == 9);
    CHECK(tune_work_class(512) == 10);
    CHECK(tune_work_class(12ull * 4096) == 16);  // 12 solves on 32^4

    // every candidate counted twice: the fastest lowest median is kept
    {
        TuneEntry e;
        const double ms[4][2] = {{2.20, 2.19}, {2.27, 2.26}, {2.35, 2.34}, {2.40, 2.42}};
        for (int round = 0; round < 2; round++)
            for (int c = 0; c < 4; c++) {
                bool timed = false;
                const int s = tune_pick(e, &timed);
                CHECK(timed);
                CHECK(s == c);  // candidates in turn
                tune_record(e, s, 4, true, ms[s][round]);
            }
        bool timed = true;
        CHECK(e.chosen == 0);
        CHECK(tune_pick(e, &timed) == 0 && !timed);
        CHECK(e.ms[0] == 2.19 && e.samples[0] == 2);
    }
    // a faster candidate later in the list wins; the decision waits for all samples
    {
        TuneEntry e;
        const double ms[4] = {3.0, 2.0, 4.0, 1.5};
        for (int c = 0; c < 4; c++) tune_record(e, c, 4, true, ms[c]);
        CHECK(e.chosen < 0);
        for (int c = 0; c < 3; c++) tune_record(e, c, 4, true, ms[c]);
        CHECK(e.chosen < 0);
        tune_record(e, 3, 4, true, 1.6);
        CHECK(e.chosen == 3);
        CHECK(e.ms[3] == 1.5);
    }
    // an uncounted chunk (a solve finished inside it) keeps the candidate for the next chunk
    {
        TuneEntry e;
        tune_record(e, 0, 4, true, 1.0);
        bool timed = false;
        CHECK(tune_pick(e, &timed) == 1);
        tune_record(e, 1, 4, false, 0.0);
        CHECK(tune_pick(e, &timed) == 1 && timed);
        CHECK(e.samples[1] == 0 && e.attempts == 2);
    }
    // a stream that never gives a countable chunk decides on the default after the cap
    {
        TuneEntry e;
        bool t0 = false;
        for (int k = 0; k < kTuneAttempts * 2 - 1; k++) tune_record(e, tune_pick(e, &t0), 2, false, 0.0);
        CHECK(e.chosen < 0);
        bool timed = false;
        tune_record(e, tune_pick(e, &timed), 2, false, 0.0);
        CHECK(e.chosen == 0);
    }
    // after the cap the fastest candidate with any sample is kept
    {
        TuneEntry e;
        tune_record(e, 0, 4, true, 2.0);
        tune_record(e, 1, 4, true, 1.0);
        for (int k = 0; k < kTuneAttempts * 4; k++) tune_record(e, 2, 4, false, 0.0);
        CHECK(e.chosen == 1);
    }
    // once decided, further records change nothing; out-of-range shapes are ignored
    {
        TuneEntry e;
        e.chosen = 2;
        tune_record(e, 0, 4, true, 0.1);
        CHECK(e.chosen == 2 && e.samples[0] == 0 && e.attempts == 0);
        TuneEntry f;
        tune_record(f, 5, 4, true, 0.1);
        tune_record(f, -1, 4, true, 0.1);
        CHECK(f.attempts == 0);
    }
    if (failures) return 1;
    std::printf("tuner logic passed\n");
    return 0;
}
