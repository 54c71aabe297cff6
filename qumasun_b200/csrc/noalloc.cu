// H|psi> without any allocation inside the call.
//
// Some callers cannot call cudaMalloc at the point where they need H|psi>:
// host programs whose device memory is owned by another framework's allocator
// (a pool that must not be bypassed), and time-critical loops that must not
// touch the allocator. qg_hamiltonian_apply_d grows a per-operator scratch
// buffer for the projector coefficients on first use; this entry point
// instead uses a fixed buffer compiled into the library (below), so the call
// itself allocates nothing. The operator handle (built earlier, outside the
// no-allocation region) supplies V and the projector tables; the caller
// passes the states in and the result buffer out.
#include <mutex>

#include "qg_internal.h"

namespace {

// Projector-coefficient scratch, [n_atoms * n_channels][ns rounded up to 16] doubles, for every
// no-allocation call on a device. 2^19 doubles = 4 MiB per device that loads
// the library, held until the process exits.
constexpr size_t kNoAllocCoefMax = size_t(1) << 19;
__device__ __align__(256) double g_noalloc_coef[kNoAllocCoefMax];

// Device address of g_noalloc_coef per device. In host code the symbol is only
// a host-side stand-in, so its address is looked up once per device with that
// device current and cached here.
constexpr int kMaxDevices = 64;
double* g_coef_addr[kMaxDevices] = {};
std::mutex g_coef_mu;

int coef_address(int device, double** out) {
    if (device < 0 || device >= kMaxDevices) return QG_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_coef_mu);
    if (!g_coef_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_coef);
        if (e != cudaSuccess) {
            qg_set_last_error("cudaGetSymbolAddress(g_noalloc_coef)", cudaGetErrorString(e), __FILE__, __LINE__);
            return QG_ERR_CUDA;
        }
        g_coef_addr[device] = static_cast<double*>(p);
    }
    *out = g_coef_addr[device];
    return QG_OK;
}

}  // namespace

extern "C" {

size_t qg_noalloc_scratch_capacity(void) { return kNoAllocCoefMax; }

int qg_hamiltonian_apply_noalloc_d(qg_hamiltonian h, int ns, const double* X, long long ldx, double* HX,
                                   long long ldhx) {
    if (!h || ns < 0 || (ns > 0 && (!X || !HX))) return QG_ERR_INVALID;
    if (ns == 0) return QG_OK;
    const long long N = h->N();
    if (ldx < N || ldhx < N) return QG_ERR_INVALID;
    if (h->gx != 0.0 || h->gy != 0.0 || h->gz != 0.0) return QG_ERR_INVALID;
    const size_t need = qg::coef_scratch_elems(h, ns);
    if (need > kNoAllocCoefMax) {
        char msg[160];
        snprintf(msg, sizeof(msg), "%d states need %zu coefficient slots, the fixed buffer holds %zu", ns, need,
                 kNoAllocCoefMax);
        qg_set_last_error("qg_hamiltonian_apply_noalloc_d", msg, __FILE__, __LINE__);
        return QG_ERR_UNSUPPORTED;
    }
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    double* coef = nullptr;
    QG_TRY(coef_address(h->ctx->device, &coef));
    return qg::apply_hamiltonian<double>(h, ns, X, ldx, HX, ldhx, coef, h->ctx->stream);
}

}  // extern "C"
