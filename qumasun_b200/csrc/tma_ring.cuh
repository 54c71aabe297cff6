// Plane-ring plumbing shared by the persistent stencil kernels (sm_100a): mbarrier
// helpers, the work decomposition and the producer lane that streams the planes of a
// block's work items into a ring of shared-memory stages with bulk async copies.
#pragma once
#include <cstdint>

#include "qg_internal.h"
#include "stencil_common.cuh"

namespace qg {
namespace ring {

constexpr int kBarBytes = 1024;  // mbarriers + control words at the front of dynamic shared memory
constexpr int kMaxStages = 16;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Plain bulk copy global -> this CTA's shared memory (no multicast), completion
// counted in bytes on `bar`. dst, src and bytes are multiples of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: gives up after ~2^31 SM clocks (about a second at 1.9 GHz).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1LL << 31)) return false;
    }
    return true;
}

struct WorkGrid {
    int tiles;   // y tiles of ty rows
    int nslab;   // z slabs
    int zslab;   // planes per slab
    int items;   // ns * tiles * nslab
};

// Producer lane: streams, for every work item of this block (item = blockIdx.x,
// blockIdx.x + gridDim.x, ...; item = (state, y tile, z slab)), the planes
// zs - R .. ze - 1 + R of its state, ty + 2R rows each (the y halo rows ride in the
// same copy, split where the tile wraps periodically in y), into ring stage
// pos % nst, pos counting planes over all items. A stage is refilled only after
// every consumer warp has arrived on its "empty" barrier. NC = 2 copies the real and
// the imaginary part of each plane into one stage. WITHV: each stage also carries, after
// the state rows, the ty rows of the local potential of that plane (the tile's own rows,
// one contiguous copy). On a wait that gives up, sets ctl[0] and the device status word
// and stops; ctl[1] = last position issued.
template <typename T, int R, int NC, bool WITHV = false>
__device__ void produce_planes(const HamArgs<T>& a, const WorkGrid& wg, int nst, int nx, T* ringp,
                               uint64_t* full, uint64_t* empty, volatile int* ctl) {
    const int ny = a.ny, nz = a.nz, ty = a.ty;
    const int rows = ty + 2 * R;
    const int comp_elems = rows * nx;
    const int stage_elems = NC * comp_elems + (WITHV ? ty * nx : 0);
    const uint32_t stage_bytes = (uint32_t)stage_elems * sizeof(T);
    const long long plane = (long long)nx * ny;
    if (a.stall) return;
    int pos = 0;
    for (int item = blockIdx.x; item < wg.items && !ctl[0]; item += gridDim.x) {
        const int slab = item % wg.nslab;
        const int tile = (item / wg.nslab) % wg.tiles;
        const int s = item / (wg.nslab * wg.tiles);
        const int y0 = tile * ty;
        const int zs = slab * wg.zslab;
        const int ze = min(nz, zs + wg.zslab);
        const T* Xs = a.X + state_offset(a, s, false);
        for (int p = zs - R; p <= ze - 1 + R; ++p, ++pos) {
            const int j = pos % nst;
            const int k = pos / nst;
            if (k > 0 && !mbar_wait(&empty[j], (uint32_t)(k - 1) & 1u)) {
                ctl[0] = 1;
                atomicExch(a.err, (int)QG_ERR_TIMEOUT);
                break;
            }
            if (ctl[0]) break;
            const long long zoff = (long long)wrap_idx(p, nz) * plane;
            T* dst = ringp + (size_t)j * stage_elems;
            mbar_expect_tx(&full[j], stage_bytes);
#pragma unroll
            for (int c = 0; c < NC; ++c) {
                const T* src = Xs + (c ? a.xim : 0) + zoff;
                int r = 0;
                while (r < rows) {
                    const int y = wrap_idx(y0 - R + r, ny);
                    const int cnt = min(rows - r, ny - y);
                    bulk_g2s(dst + (size_t)c * comp_elems + (size_t)r * nx, src + (long long)y * nx,
                             (uint32_t)(cnt * nx * sizeof(T)), &full[j]);
                    r += cnt;
                }
            }
            if constexpr (WITHV)
                bulk_g2s(dst + (size_t)NC * comp_elems, a.V + zoff + (long long)y0 * nx, (uint32_t)(ty * nx * sizeof(T)),
                         &full[j]);
            ctl[1] = pos;
        }
    }
}

// Ring stages of `stage_bytes` that fit the shared-memory budget (at least
// max(2R, R + extra) stages), or -1.
inline int ring_stages(int R, size_t stage_bytes, int extra = 2, size_t budget_kb = 200) {
    const size_t budget = budget_kb * 1024 - kBarBytes;
    int nst = (int)((budget / stage_bytes) < (size_t)kMaxStages ? budget / stage_bytes : kMaxStages);
    const int need = 2 * R > R + extra ? 2 * R : R + extra;
    return nst >= need ? nst : -1;
}

}  // namespace ring

int sm_count();

}  // namespace qg
