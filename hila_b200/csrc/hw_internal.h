// Internal host-side objects behind the opaque C-ABI handles.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/hila_b200.h"
#include "kernels.h"

namespace hw {

class Engine;

// ------------------------------------------------------------------ errors

void set_error(const char *fmt, ...);
void clear_error();

#define HW_CHECK_ARG(cond, ...)              \
    do {                                     \
        if (!(cond)) {                       \
            ::hw::set_error(__VA_ARGS__);    \
            return HW_ERR_INVALID;           \
        }                                    \
    } while (0)

#define HW_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            ::hw::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return e_ == cudaErrorMemoryAllocation ? HW_ERR_OOM : HW_ERR_CUDA;                     \
        }                                                                                          \
    } while (0)

// RAII device buffer
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    int alloc(size_t n);
    void release();
    template <typename T>
    T *as() const {
        return static_cast<T *>(ptr);
    }
};

// Sites per parity rounded up to 64 so every SoA plane starts 1 KiB aligned
// (for FP64 planes) and coalesced rows never straddle planes.
inline int padded_stride(long vh) { return (int)((vh + 63) / 64 * 64); }

}  // namespace hw

// ------------------------------------------------------------------ handles

struct hw_context {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::recursive_mutex mu;
    hw::DevBuf red_partials;  // grid-reduction partial sums
    hw::DevBuf red_ticket;    // grid-reduction arrival counters
    hw::DevBuf cg_state;      // hw::CgState
    hw::DevBuf stage;         // lexicographic staging buffer for host transfers (grow-only)
    hw::CgState *cg_state_host = nullptr;  // pinned mirror
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    hw::RedBuf red() const {
        return hw::RedBuf{red_partials.as<double>(), red_ticket.as<unsigned>()};
    }
    size_t red_capacity_doubles = 0;
    hw::Engine *engines[3] = {nullptr, nullptr, nullptr};  // batched mixed-precision engines by precision
    bool engine_profile = false;  // per-phase event timing of the engines (hw_engine_profile_enable)
};

// FP64 half-lattice field buffer
struct HalfBuf {
    hw::DevBuf buf;
    int stride = 0;
    hw::HalfF64 h() const { return hw::HalfF64{buf.as<double2>(), stride}; }
};

struct hw_lattice;

// Per-lattice FP64 solver workspace (the reference allocates r, p, Dp, DDp per
// CG call, conjugate_gradient.h:49; here they live as long as the lattice).
struct CgWorkspace {
    HalfBuf r, p, Dp, DDp, src, res;  // EVEN
    HalfBuf t;                        // ODD
    // cached graphs of the last solve
    cudaGraphExec_t init_exec = nullptr, loop_exec = nullptr;
    struct Key {
        const void *gauge = nullptr, *in = nullptr, *out = nullptr;
        double kappa = 0, acc2 = 0, diag = 1;
        int maxiter = 0, mode = 0;
        bool operator==(const Key &o) const {
            return gauge == o.gauge && in == o.in && out == o.out && kappa == o.kappa && acc2 == o.acc2 &&
                   diag == o.diag && maxiter == o.maxiter && mode == o.mode;
        }
    } key;
    bool allocated = false;
    ~CgWorkspace();
};

struct hw_field;

struct hw_lattice {
    hw_context *ctx = nullptr;
    int dims[4] = {0, 0, 0, 0};
    int tap = 1;
    long V = 0, Vh = 0;
    int stride = 0;
    hw::Geom g{};
    std::unique_ptr<CgWorkspace> ws;
    hw_field *host_b = nullptr, *host_x = nullptr;  // fields behind the host-array solve
    bool tuned = false;  // FP64 hop launch shape chosen (g.hop_variant)
    ~hw_lattice();
};

struct hw_gauge {
    hw_lattice *lat = nullptr;
    int link_format = 18;
    hw::DevBuf f64;  // FP64 planes
    hw::GaugeF64 U() const { return hw::GaugeF64{f64.as<double2>(), lat->stride, link_format == 12 ? 6 : 9}; }
    // low-precision copies for mixed-precision solves (built on first use)
    mutable hw::DevBuf f32, f16a, f16b, f32a, f32b, f16x, f16z;
};

struct hw_field {
    hw_lattice *lat = nullptr;
    HalfBuf half[2];  // [0] EVEN, [1] ODD
};

// staggered colour-vector field (staggered.cu)
struct hw_stag_field {
    hw_lattice *lat = nullptr;
    hw::DevBuf half[2];  // [0] EVEN, [1] ODD: 3 double2 planes each
};

namespace hw {
int ensure_workspace(hw_lattice *lat);
int ensure_reduction_capacity(hw_context *ctx, long nblocks);
int ensure_stage(hw_context *ctx, size_t bytes);
// pick the fastest FP64 hop launch shape for this lattice once (HW_HOP_VARIANT overrides)
int tune_hop(hw_lattice *lat, const hw_gauge *G);
// (M_s + m_h) on EVEN half fields (d = 1 + m_h), stream-ordered through the lattice's
// ODD workspace field; context lock held, workspace and hop shape ready
void eo_apply_half(const hw_gauge *G, double kappa, HalfF64 in, HalfF64 out, int sign, double d);
void destroy_engines(hw_context *ctx);
}  // namespace hw
