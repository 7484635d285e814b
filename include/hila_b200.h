/* hila_b200 — C ABI of the B200 Wilson-fermion solve path.
 *
 * Drop-in boundary for HILA's even-odd preconditioned Wilson operator and its
 * conjugate-gradient inverter.  HILA exposes these as C++ templates
 * (libraries/dirac/wilson.h, libraries/dirac/conjugate_gradient.h); every
 * entry point below names the reference interface it replaces.  The
 * C++ facade in include/hila_b200/wilson.hpp re-creates the reference's class
 * signatures on top of this ABI.
 *
 * Conventions
 *   - Every function returns an int status: HW_OK (0) or a negative HW_ERR_*
 *     code; hw_last_error() gives a message for the calling thread.
 *   - Host arrays use HILA's canonical site order: lexicographic index
 *     x + Lx*(y + Ly*(z + Lz*t)) (libraries/plumbing/lattice.cpp:559-565).
 *       spinor field: double[V][4 spin][3 colour][2]   (re, im)
 *       gauge field:  double[4 dir][V][3][3][2]       (row-major SU(3) links)
 *   - Parity masks follow HILA's Parity enum (plumbing/coordinates.h:182):
 *     HW_EVEN = 1, HW_ODD = 2, HW_ALL = 3.
 *   - Directions 0..3 = x, y, z, t.  Spinor fields are antiperiodic in t when
 *     the lattice was created with t_antiperiodic = 1 (the reference sets
 *     this per Field with set_boundary_condition(e_t, ANTIPERIODIC),
 *     applications/test_cases/test_CG.cpp:222-226); links are periodic.
 *   - Calls on one context are serialised by the context; different contexts
 *     may be used from different threads.
 */
#ifndef HILA_B200_H
#define HILA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: hw_stag_solve_request.precision / delta, hw_server_config.staggered_precision,
 *    hw_server_stats maxima, hw_engine_tuning (struct layouts changed) */
#define HW_API_VERSION 2

enum hw_status {
    HW_OK = 0,
    HW_ERR_INVALID = -1,       /* bad argument, size or handle */
    HW_ERR_OOM = -2,           /* device allocation failed */
    HW_ERR_CUDA = -3,          /* a CUDA call failed */
    HW_ERR_NOT_CONVERGED = -4, /* solve hit maxiter above tolerance */
    HW_ERR_BREAKDOWN = -5,     /* CG breakdown: p.Ap <= 0 or non-finite */
    HW_ERR_TIMEOUT = -6,       /* a bounded device wait gave up */
    HW_ERR_REJECTED = -7,      /* admission refused (over the memory budget) */
    HW_ERR_CANCELLED = -8,     /* request cancelled before completion */
    HW_ERR_NO_DEVICE = -9      /* no CUDA device / driver */
};

enum hw_parity { HW_EVEN = 1, HW_ODD = 2, HW_ALL = 3 };

/* storage precision of spinors and links */
enum hw_precision { HW_PREC_F64 = 0, HW_PREC_F32 = 1, HW_PREC_F16 = 2 };

/* link storage of the FP64 operator: 18 reals, or 12 reals with the third
 * row rebuilt as conj(row0 x row1) inside the kernel */
enum hw_link_format { HW_LINKS_18 = 18, HW_LINKS_12 = 12 };

typedef struct hw_context hw_context;
typedef struct hw_lattice hw_lattice;
typedef struct hw_gauge hw_gauge;
typedef struct hw_field hw_field;

/* ------------------------------------------------------------------ basics */

int hw_api_version(void);
/* message of the last failed call on this thread ("" if none) */
const char *hw_last_error(void);
int hw_device_count(int *count);

/* One context per GPU: owns the stream, reduction buffers and graph caches.
 * Replaces hila::initialize's device setup (libraries/plumbing/initialize.cpp). */
int hw_context_create(int device, hw_context **ctx);
/* Destroy servers, fields, gauge fields and lattices of a context before the
 * context, and fields and gauge fields of a lattice before the lattice. */
int hw_context_destroy(hw_context *ctx);
int hw_context_synchronize(hw_context *ctx);
/* The context's CUDA stream (a cudaStream_t), so callers can order their own
 * work or CUDA events with the library's.  Operator calls are stream-ordered:
 * they return once the work is enqueued; downloads and solves synchronise. */
int hw_context_stream(hw_context *ctx, void **stream);

/* Page-locked host memory for fast host<->device transfers of field arrays
 * (no reference counterpart; HILA allocates host memory with malloc). */
int hw_host_alloc(size_t bytes, void **ptr);
int hw_host_free(void *ptr);

/* Lattice geometry (lattice.setup(size), plumbing/lattice.cpp:37-104).
 * dims[0] (Lx) must be even; all dims >= 2 and even (even-odd split). */
int hw_lattice_create(hw_context *ctx, const int dims[4], int t_antiperiodic, hw_lattice **lat);
int hw_lattice_destroy(hw_lattice *lat);
int hw_lattice_volume(const hw_lattice *lat, int64_t *volume);

/* ------------------------------------------------------------------ fields */

/* Gauge field Field<SU<3,double>> U[NDIM] (the operator holds it by
 * reference, libraries/dirac/wilson.h:237, :261).  Uploads the host links once;
 * link_format selects 18- or 12-real FP64 storage for the FP64 operator.
 * Single- and half-precision copies for mixed-precision solves are made on
 * first use. */
int hw_gauge_create(hw_lattice *lat, const double *links, int link_format, hw_gauge **gauge);
int hw_gauge_destroy(hw_gauge *gauge);

/* Gauge configuration files in HILA's binary format, GaugeField::config_write /
 * config_read (gaugefield.h:196-271, Field::write / read field_io.h:128-330):
 * int64 header {394824242, 4, 144, Lx, Ly, Lz, Lt}, then the links in the host
 * layout double[4][V][3][3][2].  config_read fills a lattice whose dimensions
 * are multiples of the file's by periodic replication; errors (wrong id,
 * dimensionality, element size, dimensions, short file) return HW_ERR_INVALID
 * with the reference's message in hw_last_error().  Host only. */
int hw_gauge_config_dims(const char *path, int dims[4]);
int hw_gauge_config_write(const char *path, const int dims[4], const double *links);
int hw_gauge_config_read(const char *path, const int dims[4], double *links);

/* FP64 Wilson spinor field, Field<Wilson_vector<3,double>> (full lattice,
 * device resident, even-odd structure-of-arrays inside). */
int hw_field_create(hw_lattice *lat, hw_field **field);
int hw_field_destroy(hw_field *field);
/* copy sites of `parity` from/to a host array in the canonical layout */
int hw_field_upload(hw_field *field, const double *host, int parity);
int hw_field_download(const hw_field *field, double *host, int parity);
/* the same with the host array in HILA's even-first site order (its Field storage
 * order, lattice.cpp:171-184: the V/2 EVEN sites, then the V/2 ODD sites, each
 * double[4][3][2]): a parity is one contiguous block, so only the sites of `parity`
 * cross the bus (one copy per parity, at full rate from page-locked memory) and the
 * other parity of the host array is left as it is */
int hw_field_upload_eo(hw_field *field, const double *host, int parity);
int hw_field_download_eo(const hw_field *field, double *host, int parity);
/* field[parity] = 0 */
int hw_field_zero(hw_field *field, int parity);

/* ------------------------------------------------------------------ operators */

/* Dirac_Wilson_evenodd<SU<3,double>>::apply(in, out), wilson.h:272-279:
 * out[EVEN] = in_e - kappa^2 H^{eo} H^{oe} in_e, out[ODD] = 0. */
int hw_wilson_evenodd_apply(const hw_gauge *gauge, double kappa, const hw_field *in, hw_field *out);
/* Dirac_Wilson_evenodd::dagger(in, out), wilson.h:282-289 (sign -1) */
int hw_wilson_evenodd_dagger(const hw_gauge *gauge, double kappa, const hw_field *in, hw_field *out);

/* Hasenbusch_operator<Dirac_Wilson_evenodd>::apply / dagger, Hasenbusch.h:39-47:
 * out = (M_s + m_h) in on EVEN (sign +1 apply, -1 dagger), out[ODD] = 0.  Its
 * force is the operator's (Hasenbusch.h:49-52, hw_wilson_evenodd_force); its
 * inverse comes from the solvers with hw_cg_params.hasenbusch_mh / hw_solve_request.hasenbusch_mh. */
int hw_hasenbusch_evenodd_apply(const hw_gauge *gauge, double kappa, double mh, const hw_field *in, hw_field *out);
int hw_hasenbusch_evenodd_dagger(const hw_gauge *gauge, double kappa, double mh, const hw_field *in, hw_field *out);

/* MRE_guess(psi, chi, D, old_chi_inv), MRE_guess.h:9-88: initial guess psi for
 * the normal system (M + m_h)^dag (M + m_h) psi = chi from n earlier solutions
 * old[0..n-1]: the minimal-residual combination over their orthogonalised span
 * (real coefficients from Re<.,.> over EVEN, as the reference; the reference's
 * Gram-Schmidt and final accumulation are written as intended, not as its
 * text, which overwrites psi in its last loop).  m_h = 0 for M itself. */
int hw_mre_guess(const hw_gauge *gauge, double kappa, double mh, const hw_field *const *old, int n,
                 const hw_field *chi, hw_field *psi);

/* Dirac_Wilson_evenodd::force(chi, psi, force, sign), wilson.h:293-311 (with
 * Dirac_Wilson_calc_force, wilson.h:110-137): the derivative of
 * Re(chi^dag M_s psi) (chi, psi on EVEN) with respect to every link, as 3x3
 * complex matrices in the host link layout double[4][V][3][3][2] (the HMC adds
 * project_antihermitean(U F) to the momentum, gauge_field.h:249-256).  sign +1
 * for M (apply), -1 for M^dag.  Synchronises. */
int hw_wilson_evenodd_force(const hw_gauge *gauge, double kappa, const hw_field *chi, const hw_field *psi, int sign,
                            double *force);

/* Dirac_Wilson<SU<3,double>>::apply / dagger, wilson.h:183-192:
 * out = in - kappa H_s in over ALL sites (sign +1 apply, -1 dagger). */
int hw_wilson_apply(const hw_gauge *gauge, double kappa, int sign, const hw_field *in, hw_field *out);

/* Dirac_Wilson_hop_set (set = 1: out[parity] = -kappa H_s in) and
 * Dirac_Wilson_hop (set = 0: out[parity] -= kappa H_s in), wilson.h:15-95,
 * with the backward term gathered from x - mu.  parity is HW_EVEN or HW_ODD. */
int hw_wilson_hop(const hw_gauge *gauge, double kappa, const hw_field *in, hw_field *out, int parity, int sign,
                  int set);

/* Even-odd operator that allocates no device memory (no counterpart in the
 * reference).  For callers that may not call cudaMalloc -- code running while a
 * framework owns device memory through its own pool, code inside regions where
 * an allocation (which synchronises the device) is not allowed, hosts that
 * preallocate everything up front.  Computes out_e = M_sign in_e like
 * hw_wilson_evenodd_apply (sign +1 apply, -1 dagger) from device arrays in the
 * library's even-odd layout: links = ((parity*4 + dir)*planes + k)*stride + i
 * double2 planes (planes 9 for link_format 18, 6 for 12); in_even / out_even =
 * 12 double2 planes of `stride` sites (component 3*spin + colour).  The odd
 * temporary comes from a fixed 6 MiB device array inside the library, so the
 * lattice may have at most 32768 sites per parity (a 16^4 lattice); larger
 * lattices are rejected with HW_ERR_INVALID.  Stream-ordered on `stream`
 * (a cudaStream_t, NULL = default stream) of the current device.  The first
 * call on a device looks up the array's device address; make that first call
 * before any stream capture.  Calls share the array: calls that overlap on the
 * GPU (other streams or threads on the same device) race. */
int hw_wilson_evenodd_apply_noalloc(const int dims[4], int t_antiperiodic, double kappa, int sign,
                                    const double *links, int link_format, const double *in_even, double *out_even,
                                    int stride, void *stream);

/* ------------------------------------------------------------------ solver */

typedef struct hw_cg_params {
    double accuracy;     /* relative accuracy (CG_DEFAULT_ACCURACY = 1e-12, conjugate_gradient.h:16) */
    int maxiters;        /* CG_DEFAULT_MAXITERS = 10000 (conjugate_gradient.h:15) */
    int precision;       /* HW_PREC_F64: plain FP64 CG; HW_PREC_F32 / HW_PREC_F16: mixed precision
                            with FP64 reliable updates, solution accumulation and dot products */
    double delta;        /* reliable-update trigger: recompute the FP64 residual when the iterated
                            residual fell by this factor (mixed precision only; 0 = default 0.1) */
    int true_residual;   /* 1: stop only when the explicitly recomputed FP64 residual meets
                            accuracy; 0: reference stopping rule on the iterated residual */
    int use_graph;       /* 1: device-resident iteration in a CUDA graph (default); 0: host loop */
    double hasenbusch_mh; /* m_h of the Hasenbusch operator M + m_h (Hasenbusch.h:16-52); 0: M itself */
} hw_cg_params;

typedef struct hw_cg_result {
    int status;             /* HW_OK, HW_ERR_NOT_CONVERGED or HW_ERR_BREAKDOWN */
    int iterations;         /* CG iterations (inner iterations in mixed precision) */
    int reliable_updates;   /* FP64 residual recomputations */
    int restarts;           /* continuations after an explicit residual check */
    double rr_relative;     /* |r|^2/|in|^2 of the iterated residual, as the reference prints
                               it (conjugate_gradient.h:103) */
    double true_residual;   /* |b - A x| / |b| recomputed in FP64 */
    double seconds;         /* device time of the solve */
    int kernel_launches;    /* CUDA kernels the solve launched (graph nodes included) */
} hw_cg_result;

/* fill params with the reference defaults (accuracy 1e-12, maxiters 10000, FP64) */
void hw_cg_params_default(hw_cg_params *params);

/* CG<Dirac_Wilson_evenodd<SU<3,double>>>::apply(in, out),
 * conjugate_gradient.h:46-104: solves (M^dagger M) out = in on EVEN sites;
 * `out` holds the initial guess on entry. */
int hw_cg_solve(const hw_gauge *gauge, double kappa, const hw_field *in, hw_field *out,
                const hw_cg_params *params, hw_cg_result *result);
/* CG<Dirac_Wilson>::apply (conjugate_gradient.h:46-104 on the unpreconditioned operator,
 * wilson.h:146-201, as test_CG.cpp:127-182 uses it): M^dag M out = in on ALL sites,
 * out the initial guess, FP64 (params->precision must be HW_PREC_F64; NULL: defaults);
 * stops when |r|^2 < accuracy^2 |in|^2 (with true_residual set, also on the recomputed
 * |in - M^dag M out| / |in|, which result->true_residual reports). */
int hw_wilson_cg_solve(const hw_gauge *gauge, double kappa, const hw_field *in, hw_field *out,
                       const hw_cg_params *params, hw_cg_result *result);

/* Solve M x = b on EVEN sites (M = Dirac_Wilson_evenodd) by CG on the normal
 * equations with source M^dagger b — the D (D^dag D)^{-1} D^dag pattern of
 * test_CG.cpp:254-256.  result->true_residual = |b - M x| / |b|; with
 * params->true_residual = 1 the solve continues until that is <= accuracy. */
int hw_wilson_evenodd_solve(const hw_gauge *gauge, double kappa, const hw_field *b, hw_field *x,
                            const hw_cg_params *params, hw_cg_result *result);

/* Same solve from and to host arrays (canonical layout, EVEN sites used):
 * uploads b, solves, downloads x.  Host-to-device and device-to-host copies
 * are part of the call. */
int hw_wilson_evenodd_solve_host(const hw_gauge *gauge, double kappa, const double *b_host, double *x_host,
                                 const hw_cg_params *params, hw_cg_result *result);

/* ------------------------------------------------------------------ batches */

/* One solve of M x = b (EVEN sites) inside a batch. */
typedef struct hw_solve_request {
    const hw_gauge *gauge; /* gauge field (selects the lattice) */
    double kappa;
    const hw_field *b;     /* right-hand side */
    hw_field *x;           /* solution; holds the initial guess on entry */
    double accuracy;       /* stop when |b - M x| / |b| <= accuracy (FP64, recomputed) */
    int maxiters;
    double hasenbusch_mh;  /* solve (M + m_h) x = b instead (Hasenbusch.h:16-52); 0: M */
} hw_solve_request;

/* Many right-hand sides on many lattices at once (no reference counterpart:
 * HILA solves one source per CG<Op>::apply call).  Mixed precision (FP32, or
 * FP16 with per-site scale) inner CG with FP64 reliable updates, solution
 * accumulation and dot products; `delta` is the reliable-update factor
 * (<= 0: 0.1).  Every CG phase of all admitted solves runs in one kernel
 * launch; up to 16 solves per lattice and 64 in total run at a time, the rest
 * are admitted as earlier ones finish.  results[k] receives request k's
 * outcome; each solve gives bitwise the same result alone and in a batch. */
int hw_batch_solve(hw_context *ctx, int precision, double delta, const hw_solve_request *requests, int n,
                   hw_cg_result *results);

/* ------------------------------------------------------------------ serving */

/* A solve server over one context (no reference counterpart: HILA has no
 * serving layer).  Gauge fields stay device resident; requests (gauge, kappa,
 * 1..16 sources, accuracy) are queued by any thread and run by a server thread
 * with continuous batching on the mixed-precision engine: between chunks of
 * `chunk_iters` CG iterations it retires finished solves and admits waiting
 * requests while others keep iterating, as long as the requests' solve memory
 * fits `hbm_budget_bytes`.  Each solve's result is bitwise the same alone and
 * in any mix. */
typedef struct hw_server hw_server;

typedef struct hw_server_config {
    int precision;            /* HW_PREC_F16 (default) or HW_PREC_F32 inner solves */
    double delta;             /* reliable-update factor (<= 0: 0.005 for FP16, 1e-5 for FP32) */
    size_t hbm_budget_bytes;  /* device memory for solve slots (0: 80% of free memory at creation) */
    int chunk_iters;          /* CG iterations between admission points (<= 0: 8) */
    size_t host_pool_bytes;   /* idle page-locked host buffers the server keeps for reuse (0: 16 GiB) */
    int staggered_precision;  /* staggered requests: HW_PREC_F64 (0, default) or HW_PREC_F16 (FP16 inner
                                 iterations, FP64 reliable updates, factor 0.05; needs precision F16) */
} hw_server_config;

typedef struct hw_request_result {
    int status;               /* HW_OK, HW_ERR_NOT_CONVERGED, HW_ERR_BREAKDOWN, HW_ERR_CANCELLED, HW_ERR_REJECTED */
    int nrhs;
    int iterations;           /* largest iteration count over the request's sources */
    int reliable_updates;     /* largest over the sources */
    double true_residual;     /* largest |b - M x| / |b| over the sources (FP64) */
    double latency_seconds;   /* submit -> result available */
    double queue_seconds;     /* submit -> admitted */
    uint64_t admit_chunk;     /* chunks the server had launched when the request was admitted ... */
    uint64_t retire_chunk;    /* ... and when it retired: a request admitted while another one's
                                 [admit_chunk, retire_chunk) interval was open ran beside it */
} hw_request_result;

typedef struct hw_server_stats {
    uint64_t submitted, completed, rejected, cancelled, running, queued;
    size_t bytes_in_use, bytes_budget;
    double latency_p50_seconds, latency_p99_seconds;  /* over completed requests */
    uint64_t solves_completed;                         /* sources, not requests */
    uint64_t chunks;                                   /* chunk graphs launched */
    uint64_t kernel_launches;                          /* kernels those chunks ran */
    double seconds_admit;                              /* server-thread wall time admitting requests */
    double seconds_run;                                /* ... launching chunks and reading slot states */
    double seconds_retire;                             /* ... copying solutions out and retiring */
    /* the longest single pass of each server-thread section; submissions wait for the
     * server lock while one runs (admission, chunk launch, retirement) */
    double max_admit_seconds, max_launch_seconds, max_retire_seconds;
} hw_server_stats;

int hw_server_create(hw_context *ctx, const hw_server_config *config, hw_server **server);
int hw_server_destroy(hw_server *server);
/* register a gauge field with the server (it must outlive the server) */
int hw_server_add_gauge(hw_server *server, const hw_gauge *gauge, int *gauge_id);
/* queue M x = b for nrhs host sources (canonical layout, EVEN sites used);
 * the sources are copied before the call returns */
int hw_server_submit(hw_server *server, int gauge_id, double kappa, int nrhs, const double *const *sources,
                     double accuracy, int maxiters, uint64_t *request_id);
/* queue M x = b for nrhs host sources in HILA's even-first site order (the order of
 * its Field storage, lattice.cpp:171-184: the V/2 EVEN sites first, each site
 * double[4][3][2]); only the EVEN half of each source is read and only the EVEN half
 * of each solution written.  Page-locked arrays (cudaHostAlloc / cudaHostRegister)
 * are read and written by DMA directly: the caller keeps them valid and unread until
 * the request's wait returns.  Pageable sources are copied before the call returns;
 * pageable solutions are filled by hw_server_wait.  `solutions` (or an entry) may be
 * NULL: the solution is then copied by hw_server_wait into its `solutions` argument
 * (EVEN half, even-first order) if one is given there. */
int hw_server_submit_eo(hw_server *server, int gauge_id, double kappa, int nrhs, const double *const *sources,
                        double *const *solutions, double accuracy, int maxiters, uint64_t *request_id);
/* queue M x = b for nrhs device fields of the gauge field's lattice (the form HILA's
 * fermion code holds, hmc/fermion_field.h:90-103): the engine reads the EVEN half of
 * sources[k] and accumulates the solution in the EVEN half of solutions[k], whose
 * content on submit is the initial guess (zero it for none).  Nothing is copied; the
 * caller leaves the fields alone until the request's wait returns. */
int hw_server_submit_fields(hw_server *server, int gauge_id, double kappa, int nrhs, const hw_field *const *sources,
                            hw_field *const *solutions, double accuracy, int maxiters, uint64_t *request_id);
/* queue the staggered solves M x = b (dirac_staggered_evenodd, staggered.h:193-279, at
 * `mass`) for nrhs device colour-vector fields of the gauge field's lattice, in place as
 * hw_server_submit_fields (solutions[k] holds the initial guess); FP64, batched with the
 * server's other requests.  hw_stag_field: a staggered field (operator section below). */
typedef struct hw_stag_field hw_stag_field;
int hw_server_submit_staggered(hw_server *server, int gauge_id, double mass, int nrhs,
                               const hw_stag_field *const *sources, hw_stag_field *const *solutions,
                               double accuracy, int maxiters, uint64_t *request_id);
/* wait up to timeout_seconds (< 0: forever) for a request; on completion copy
 * the solutions of an hw_server_submit request (canonical layout, ODD sites zero)
 * into solutions[0..nrhs-1] (solutions or an entry may be NULL; field requests have
 * their solutions in place, and hw_server_submit_eo requests use it only for the
 * entries they were not given) and fill *result.  HW_ERR_TIMEOUT if still running.  A finished request is forgotten
 * after its wait. */
int hw_server_wait(hw_server *server, uint64_t request_id, double *const *solutions, double timeout_seconds,
                   hw_request_result *result);
/* cancel a queued or running request (its slots are freed at the next chunk) */
int hw_server_cancel(hw_server *server, uint64_t request_id);
int hw_server_stats_get(hw_server *server, hw_server_stats *stats);

/* ------------------------------------------------------------------ staggered fermions */

/* Field<SU_vector<3,double>> for staggered fermions (libraries/dirac/staggered.h):
 * host layout double[V][3][2] (colour-vector complex, lexicographic). */
/* hw_stag_field is declared with the serving entry points above */
int hw_stag_field_create(hw_lattice *lat, hw_stag_field **field);  /* zero-filled */
int hw_stag_field_destroy(hw_stag_field *field);
int hw_stag_field_upload(hw_stag_field *field, const double *host, int parity);
/* sites of the parities not requested come back as zero */
int hw_stag_field_download(const hw_stag_field *field, double *host, int parity);
/* zero the sites of `parity` (the field's memory stays allocated) */
int hw_stag_field_zero(hw_stag_field *field, int parity);

/* dirac_staggered_evenodd<SU<3,double>>::apply / dagger, staggered.h:224-242:
 * out[EVEN] = m in_e + D_eo (1/m) D_oe in_e with D = 0.5 s sum_mu eta_mu (U fwd -
 * U^dag bwd) (staggered.h:48-68, eta as staggered.h:14-28 codes it); out[ODD]
 * keeps (1/m) D_oe in_e as the reference leaves it.  Stream-ordered. */
int hw_staggered_evenodd_apply(const hw_gauge *gauge, double mass, const hw_stag_field *in, hw_stag_field *out);
int hw_staggered_evenodd_dagger(const hw_gauge *gauge, double mass, const hw_stag_field *in, hw_stag_field *out);
/* dirac_staggered_evenodd::force(chi, psi, force, sign), staggered.h:246-265 and
 * :70-86, in the host link layout double[4][V][3][3][2].  Synchronises. */
int hw_staggered_evenodd_force(const hw_gauge *gauge, double mass, const hw_stag_field *chi, const hw_stag_field *psi,
                               int sign, double *force);
/* One staggered solve inside a batch (dirac_staggered_evenodd, staggered.h:193-279). */
typedef struct hw_stag_solve_request {
    const hw_gauge *gauge;     /* gauge field (selects the lattice) */
    double mass;
    const hw_stag_field *in;   /* right-hand side (EVEN) */
    hw_stag_field *out;        /* solution (EVEN); holds the initial guess on entry */
    double accuracy;           /* stop on the FP64-recomputed residual (below) <= accuracy */
    int maxiters;
    int normal;                /* 1: M^dag M out = in, CG<Op>::apply semantics (conjugate_gradient.h:46-104),
                                  residual |in - M^dag M out| / |in|; 0: M out = in, residual
                                  |in - M out| / |in| (CG on M^dag M with source M^dag in) */
    int precision;             /* HW_PREC_F64 (0): FP64 throughout; HW_PREC_F16: inner iterations in
                                  FP32 arithmetic on FP16 fields with FP64 reliable updates */
    double delta;              /* HW_PREC_F16: reliable-update factor (<= 0: 0.05) */
} hw_stag_solve_request;
/* Many staggered solves on many lattices at once, on the same batched engine as the
 * Wilson solves (no reference counterpart: HILA runs one CG<Op>::apply per source):
 * CG in one kernel launch per phase for all admitted solves, up to 16 per lattice and
 * 64 in total at a time, in FP64 or mixed precision per request (the FP64 solution, the
 * reliable updates and the convergence test always in FP64); results[k] is request k's
 * outcome (iterations, recomputed FP64 true residual); each solve gives bitwise the
 * same result alone and in any batch, also beside Wilson solves of the same engine. */
int hw_staggered_batch_solve(hw_context *ctx, const hw_stag_solve_request *requests, int n, hw_cg_result *results);
/* CG<dirac_staggered_evenodd>::apply, conjugate_gradient.h:46-104: M^dag M out = in
 * on EVEN, out the initial guess; FP64 (params->precision must be HW_PREC_F64);
 * result reports the recomputed |in - M^dag M out| / |in|. */
int hw_staggered_cg_solve(const hw_gauge *gauge, double mass, const hw_stag_field *in, hw_stag_field *out,
                          const hw_cg_params *params, hw_cg_result *result);

/* ------------------------------------------------------------------ profiling */

/* Device time per phase of the batched mixed-precision engines behind
 * hw_cg_solve / hw_wilson_evenodd_solve (FP32, FP16) and hw_batch_solve, from
 * CUDA events around every phase launch (the reference has no counterpart; it
 * times whole calls, bench_fermion.cpp:95-120).  While enabled, iterations run
 * from a host loop that synchronises after each one, so solves are slower; the
 * phase times are those of the same kernels.  Phases 0..11: P1 t = H p, P2
 * Dp = M p and |Dp|^2, P3 t = H^dag Dp, P4 r -= alpha M^dag Dp, y += alpha p,
 * |r|^2; the reliable update R1 x += y, R2 and R3 s = b - M x in FP64, then
 * r = M^dag s by R4, R5 (FP64, normal system) or R4L, R5L (low precision,
 * M x = b); P5 p = r + beta p. */
#define HW_ENGINE_PHASES 12
/* Work units of a phase, summed over its launches that had work:
 *   [0] sites x solves that ran the phase's main form;
 *   [1] sites x solves of its alternate form: R1 of a normal-equation solve (y also
 *       cleared), R3 of a first reliable update from x = 0 (no hop), P5 of a first
 *       iteration (p = r, p not read);
 *   [2] sites whose links the launch read (once per site, shared by the solves);
 *   [3] R3 of a normal-equation solve (s = M x stored in FP64).
 * Multiplied by the bytes each unit moves they give a launch's algorithmic bytes. */
#define HW_ENGINE_WORK_KINDS 4
typedef struct hw_engine_profile {
    int launches[HW_ENGINE_PHASES]; /* launches that had work */
    double ms[HW_ENGINE_PHASES];    /* their summed device time */
    unsigned long long work[HW_ENGINE_PHASES][HW_ENGINE_WORK_KINDS];
} hw_engine_profile;
/* enabling resets the counters of the context's engines */
int hw_engine_profile_enable(hw_context *ctx, int enable);
/* counters of the engine of one precision (HW_PREC_F32 / HW_PREC_F16); zeros if it has not run */
int hw_engine_profile_get(hw_context *ctx, int precision, hw_engine_profile *out);

/* The launch-shape tuner of the batched engines (no reference counterpart).  The inner
 * phases have launch shapes that round every product and sum alike: two solves per
 * thread in packed FP32 or one, each with tiles taken from a counter or in a fixed
 * order.  An engine times them on chunks of real iterations of the running solves
 * (median device time per iteration of P1..P4 and P5) and keeps the fastest per work
 * class, the bit length of the sum over the running Wilson solves of their lattice's
 * 128-site tiles (classes below 10, about one wave of blocks, run the default shape
 * untimed).  A solve's result does not depend on the shape.  HW_ENGINE_TUNE=0
 * turns the tuner off; HW_ENGINE_VARIANT or HW_ENGINE_SCHED force a shape instead. */
#define HW_TUNE_MAX_SHAPES 4
typedef struct hw_engine_tuning {
    int work_class;
    int nshapes;                                  /* candidates of this engine */
    int variant[HW_TUNE_MAX_SHAPES];              /* launch shape (HW_ENGINE_VARIANT values) */
    int dynamic_order[HW_TUNE_MAX_SHAPES];        /* 1: tiles from a counter; 0: fixed order */
    double ms_per_iteration[HW_TUNE_MAX_SHAPES];  /* lowest median seen; 0: not timed yet */
    int samples[HW_TUNE_MAX_SHAPES];              /* timed chunks */
    int chosen;                                   /* index of the kept shape; -1 while timing */
} hw_engine_tuning;
/* Up to max entries, by increasing work class, of the engine of one precision; *n is the
 * number written (0 if the engine has not run or the tuner is off). */
int hw_engine_tuning_get(hw_context *ctx, int precision, hw_engine_tuning *out, int max, int *n);

/* ------------------------------------------------------------------ inputs */

/* Seeded synthetic inputs (no reference counterpart beyond hila::seed_random
 * + SU::random / gaussian_random; plumbing/random.cpp:60-70,187-199,
 * datatypes/sun_matrix.h:137-196,480-560, matrix.h:3289-3309):
 *   links  U = reunitarize(exp(eps * A)), A anti-Hermitian traceless from
 *          8 Gaussian algebra coefficients of variance 2 per link
 *   spinor every complex entry from Box-Muller (re, im each N(0,1)) on the
 *          sites of parity_mask, zero elsewhere. */
int hw_generate_links(const int dims[4], double eps, uint64_t seed, double *links);
int hw_generate_spinor(const int dims[4], uint64_t seed, int parity_mask, double *spinor);

#ifdef __cplusplus
}
#endif

#endif /* HILA_B200_H */
