// Context, status strings and error reporting of the C ABI.
#include <cstring>
#include <mutex>
#include <string>

#include "qg_internal.h"
#include <cublas_v2.h>
#include <cusolverDn.h>

static thread_local std::string g_last_error;

void qg_set_last_error(const char* what, const char* msg, const char* file, int line) {
    char buf[512];
    snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, msg, file, line);
    g_last_error = buf;
}

extern "C" {

const char* qg_last_error(void) { return g_last_error.c_str(); }

int qg_version(void) { return QG_API_VERSION; }

const char* qg_status_string(int status) {
    switch (status) {
        case QG_OK: return "ok";
        case QG_ERR_INVALID: return "invalid argument";
        case QG_ERR_CUDA: return "CUDA error";
        case QG_ERR_NOMEM: return "device out of memory";
        case QG_ERR_CHOLESKY: return "Gram matrix not positive definite";
        case QG_ERR_TIMEOUT: return "bounded device wait timed out";
        case QG_ERR_NONFINITE: return "non-finite value";
        case QG_ERR_UNSUPPORTED: return "unsupported shape or option";
        case QG_ERR_LIBRARY: return "CUDA library error";
        case QG_ERR_NOT_CONVERGED: return "not converged within the iteration limit";
        default: return "unknown status";
    }
}

int qg_context_create(int device, qg_context* out) {
    if (!out) return QG_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    QG_CUDA_TRY(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(device));
    qg_context c = new qg_context_s();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return QG_ERR_CUDA;
    }
    c->stream = c->own_stream;
    if (cudaMalloc(&c->dev_status, sizeof(int)) != cudaSuccess ||
        cudaMemset(c->dev_status, 0, sizeof(int)) != cudaSuccess) {
        cudaStreamDestroy(c->own_stream);
        delete c;
        return QG_ERR_CUDA;
    }
    *out = c;
    return QG_OK;
}

void qg_release_libraries(qg_context c) {
    if (c->blas) cublasDestroy(static_cast<cublasHandle_t>(c->blas));
    if (c->solver) cusolverDnDestroy(static_cast<cusolverDnHandle_t>(c->solver));
    c->blas = nullptr;
    c->solver = nullptr;
}

int qg_context_destroy(qg_context c) {
    if (!c) return QG_ERR_INVALID;
    if (c->live_hamiltonians > 0) return QG_ERR_INVALID;
    cudaSetDevice(c->device);
    qg_release_libraries(c);
    qg_release_gram_cache(c);
    if (c->stream) cudaStreamSynchronize(c->stream);
    c->small.release();
    if (c->own_stream) {
        cudaStreamSynchronize(c->own_stream);
        cudaStreamDestroy(c->own_stream);
    }
    if (c->dev_status) cudaFree(c->dev_status);
    delete c;
    return QG_OK;
}

int qg_context_set_stream(qg_context c, void* stream) {
    if (!c) return QG_ERR_INVALID;
    c->stream = static_cast<cudaStream_t>(stream);
    return QG_OK;
}

int qg_context_synchronize(qg_context c) {
    if (!c) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(c->device));
    QG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return qg_context_take_device_status(c);
}

int qg_context_take_device_status(qg_context c) {
    if (!c) return QG_ERR_INVALID;
    int v = 0;
    QG_CUDA_TRY(cudaMemcpy(&v, c->dev_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (v != 0) QG_CUDA_TRY(cudaMemset(c->dev_status, 0, sizeof(int)));
    return v;
}


}  // extern "C"
