// Even-odd Wilson operator for callers that cannot allocate device memory.
//
// Some callers of this library may not call cudaMalloc: code that runs while a
// framework owns all device memory through its own pool allocator, code inside
// a region where allocation is forbidden (allocation synchronises the device and
// can deadlock or break an enclosing stream capture), or small embedded hosts
// that preallocate everything at start-up.  hw_wilson_evenodd_apply needs a
// temporary odd-parity spinor field, which the normal path allocates once per
// lattice.  The entry point below takes that temporary from a fixed array in
// the library's own device data instead, so it allocates nothing: the caller
// passes the links and both spinor fields as device pointers.
//
// The array holds one FP64 half spinor of at most kNoAllocMaxSites sites per
// parity (a 16^4 lattice): 12 x 32768 x 16 bytes = 6 MiB, kept by every GPU that
// loads the library until the process exits.  All calls share it, so calls
// that overlap on the GPU (different streams, or different host threads on the
// same device) race on it; calls on one stream are ordered and safe.  Every
// scratch site that is read is first written by the same call, so nothing in
// the array has to start at zero.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "hw_internal.h"

namespace hw {
namespace {

constexpr int kNoAllocMaxSites = 32768;  // sites per parity
constexpr int kNoAllocMaxDevices = 64;

// the temporary odd-parity half spinor: 12 planes of kNoAllocMaxSites double2
static __device__ __align__(256) double2 g_noalloc_odd[12 * kNoAllocMaxSites];

std::mutex g_noalloc_mu;
double2 *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device.  Host code must
// not use the symbol itself (it is a host-side stand-in): the address comes
// from cudaGetSymbolAddress, once per device, with that device current.
int noalloc_scratch(double2 **out) {
    int dev = 0;
    HW_CUDA(cudaGetDevice(&dev));
    HW_CHECK_ARG(dev >= 0 && dev < kNoAllocMaxDevices, "device %d beyond the %d supported", dev, kNoAllocMaxDevices);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_odd);
        if (e != cudaSuccess || !p) {
            set_error("cudaGetSymbolAddress(scratch) failed on device %d: %s", dev, cudaGetErrorString(e));
            return HW_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = static_cast<double2 *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return HW_OK;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

}  // namespace
}  // namespace hw

using namespace hw;

extern "C" int hw_wilson_evenodd_apply_noalloc(const int dims[4], int t_antiperiodic, double kappa, int sign,
                                               const double *links, int link_format, const double *in_even,
                                               double *out_even, int stride, void *stream) {
    HW_CHECK_ARG(dims && links && in_even && out_even, "null argument");
    // the running product is checked after every factor, so it never exceeds
    // 2 * kNoAllocMaxSites * 2^31 and cannot overflow
    long V = 1;
    for (int d = 0; d < 4; d++) {
        HW_CHECK_ARG(dims[d] >= 2 && dims[d] % 2 == 0, "dims[%d] = %d: every extent must be even and >= 2", d,
                     dims[d]);
        V *= dims[d];
        HW_CHECK_ARG(V <= 2L * kNoAllocMaxSites,
                     "lattice has more than %d sites per parity; the allocation-free operator supports at most "
                     "%d (a 16^4 lattice) -- use hw_wilson_evenodd_apply",
                     kNoAllocMaxSites, kNoAllocMaxSites);
    }
    const long Vh = V / 2;
    HW_CHECK_ARG(stride >= Vh, "stride %d is smaller than the %ld sites per parity", stride, Vh);
    HW_CHECK_ARG(sign == 1 || sign == -1, "sign must be +1 (apply) or -1 (dagger)");
    HW_CHECK_ARG(link_format == 18 || link_format == 12, "link_format must be 18 or 12");
    HW_CHECK_ARG(aligned16(links) && aligned16(in_even) && aligned16(out_even),
                 "device arrays must be 16-byte aligned");
    double2 *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc != HW_OK) return rc;

    Geom g{};
    geom_setup(g, dims, t_antiperiodic);
    const GaugeF64 U{reinterpret_cast<const double2 *>(links), stride, link_format == 12 ? 6 : 9};
    const HalfF64 in{const_cast<double2 *>(reinterpret_cast<const double2 *>(in_even)), stride};
    const HalfF64 out{reinterpret_cast<double2 *>(out_even), stride};
    const HalfF64 t{scratch, kNoAllocMaxSites};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // t_o = H^{oe}_s in_e ; out_e = in_e - kappa^2 H^{eo}_s t_o  (wilson.h:272-289)
    launch_hop_scale(g, U, 1, sign, in, t, 1.0, nullptr, s);
    launch_hop_xpay(g, U, 0, sign, t, in, out, -kappa * kappa, nullptr, nullptr, s);
    HW_CUDA(cudaGetLastError());
    return HW_OK;
}
