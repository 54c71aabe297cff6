// FD stencil + local potential, H psi = V psi - 1/2 Lap psi, as a persistent,
// TMA-staged, warp-specialised kernel (sm_100a).
//
//  * one block per SM loops over work items (state, y tile of ty full x-rows,
//    z slab); the plane ring and its mbarrier phases run on across items, so the
//    pipeline never drains between items;
//  * warp 0 is the producer: one lane streams every plane an item needs (ty + 2R
//    rows: the y halo rows ride in the same copy, split where the tile wraps
//    periodically in y) into a ring of `nst` shared-memory stages with bulk async
//    copies (cp.async.bulk), completion counted on a "full" mbarrier per stage;
//  * the other warps are consumers: each thread owns PX consecutive x-points
//    (one 16-byte vector) of one row, keeps their 2R+1 z-values in registers
//    (filled from the ring), reads x and y neighbours from the stage of the
//    current plane with 16-byte shared loads (x wraps by index), prefetches V
//    R planes ahead into registers, and writes H psi with 16-byte stores;
//  * a consumer warp releases a stage by arriving on its "empty" mbarrier once
//    its reads of that plane are done; the producer refills a stage only after
//    every consumer warp released it. No block-wide barrier per plane.
// Every mbarrier wait is bounded (~2^31 SM clocks); on timeout the thread
// records QG_ERR_TIMEOUT in the device status word and the block winds down:
// consumers stop, the producer stops issuing, and after a final block barrier
// the producer lane waits (bounded) for its copies still in flight.
#include <atomic>
#include <cstdint>

#include "qg_internal.h"
#include "stencil_common.cuh"

namespace qg {
namespace {

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

template <typename T, int PX>
struct VecOf;
template <>
struct VecOf<double, 2> { using type = double2; };
template <>
struct VecOf<float, 4> { using type = float4; };

template <typename T, int PX>
union Vec {
    typename VecOf<T, PX>::type v;
    T e[PX];
};

// Laplacian of one point from its neighbours: xm[d]/xp[d] at x -/+ (d+1), same for y, z.
// Groupings follow Laplasian{2nd,4th,6th,8th}_halo_f (GridDifference2nd.h:1027-1031,
// 4th.h:528-530, 6th.h:425-429, 8th.h:141-145).
template <typename T, int ORDER>
__device__ __forceinline__ T lap_point(T c, const T* xm, const T* xp, const T* ym, const T* yp, const T* zm,
                                       const T* zp, const HamArgs<T>& a) {
    if constexpr (ORDER == 2) {
        return a.cx[0] * (xp[0] + xm[0] - T(2) * c) + a.cy[0] * (yp[0] + ym[0] - T(2) * c) +
               a.cz[0] * (zp[0] + zm[0] - T(2) * c);
    } else if constexpr (ORDER == 4) {
        return a.cx[2] * ((xp[2] + xm[2]) - T(54) * (xp[1] + xm[1]) + T(783) * (xp[0] + xm[0]) - T(1460) * c) +
               a.cy[2] * ((yp[2] + ym[2]) - T(54) * (yp[1] + ym[1]) + T(783) * (yp[0] + ym[0]) - T(1460) * c) +
               a.cz[2] * ((zp[2] + zm[2]) - T(54) * (zp[1] + zm[1]) + T(783) * (zp[0] + zm[0]) - T(1460) * c);
    } else if constexpr (ORDER == 6) {
        T d = a.c0 * c;
        d += a.cx[2] * (xp[2] + xm[2]) + a.cx[1] * (xp[1] + xm[1]) + a.cx[0] * (xp[0] + xm[0]);
        d += a.cy[2] * (yp[2] + ym[2]) + a.cy[1] * (yp[1] + ym[1]) + a.cy[0] * (yp[0] + ym[0]);
        d += a.cz[2] * (zp[2] + zm[2]) + a.cz[1] * (zp[1] + zm[1]) + a.cz[0] * (zp[0] + zm[0]);
        return d;
    } else {
        T d = a.c0 * c;
        d += a.cx[3] * (xp[3] + xm[3]) + a.cx[2] * (xp[2] + xm[2]) + a.cx[1] * (xp[1] + xm[1]) + a.cx[0] * (xp[0] + xm[0]);
        d += a.cy[3] * (yp[3] + ym[3]) + a.cy[2] * (yp[2] + ym[2]) + a.cy[1] * (yp[1] + ym[1]) + a.cy[0] * (yp[0] + ym[0]);
        d += a.cz[3] * (zp[3] + zm[3]) + a.cz[2] * (zp[2] + zm[2]) + a.cz[1] * (zp[1] + zm[1]) + a.cz[0] * (zp[0] + zm[0]);
        return d;
    }
}

// g.grad of one point with the first derivative of the FD order: 8th (672, -168, 32, -3)/840h,
// 6th (45, -9, 1)/60h, 2nd 1/2h, grouped as in LaplasianKpoint{8th,6th,2nd}_halo_f
// (GridDifferenceKpoint8th.h:18-122, 6th.h:19-107, 2nd.h:19-92); the factor 2*coef and g
// are folded into a.dx/dy/dz.
template <typename T, int ORDER>
__device__ __forceinline__ T der_point(const T* xm, const T* xp, const T* ym, const T* yp, const T* zm,
                                       const T* zp, const HamArgs<T>& a) {
    if constexpr (ORDER == 2) {
        T g = a.dx[0] * (xp[0] - xm[0]);
        g += a.dy[0] * (yp[0] - ym[0]);
        g += a.dz[0] * (zp[0] - zm[0]);
        return g;
    } else if constexpr (ORDER == 6) {
        T g = a.dx[2] * (xp[2] - xm[2]) + a.dx[1] * (xp[1] - xm[1]) + a.dx[0] * (xp[0] - xm[0]);
        g += a.dy[2] * (yp[2] - ym[2]) + a.dy[1] * (yp[1] - ym[1]) + a.dy[0] * (yp[0] - ym[0]);
        g += a.dz[2] * (zp[2] - zm[2]) + a.dz[1] * (zp[1] - zm[1]) + a.dz[0] * (zp[0] - zm[0]);
        return g;
    } else {
        T g = a.dx[3] * (xp[3] - xm[3]) + a.dx[2] * (xp[2] - xm[2]) + a.dx[1] * (xp[1] - xm[1]) + a.dx[0] * (xp[0] - xm[0]);
        g += a.dy[3] * (yp[3] - ym[3]) + a.dy[2] * (yp[2] - ym[2]) + a.dy[1] * (yp[1] - ym[1]) + a.dy[0] * (yp[0] - ym[0]);
        g += a.dz[3] * (zp[3] - zm[3]) + a.dz[2] * (zp[2] - zm[2]) + a.dz[1] * (zp[1] - zm[1]) + a.dz[0] * (zp[0] - zm[0]);
        return g;
    }
}

// -1/2 (Lap - g^2) of one point for complex k-point states: orders 6 and 8 as lap_point
// (a.c0 carrying -coef g^2); order 2 grouped as LaplasianKpoint2nd_halo_f
// (GridDifferenceKpoint2nd.h:69-72), c0 p + cx (p+x + p-x) + cy (..) + cz (..).
template <typename T, int ORDER>
__device__ __forceinline__ T lap_point_k(T c, const T* xm, const T* xp, const T* ym, const T* yp, const T* zm,
                                         const T* zp, const HamArgs<T>& a) {
    if constexpr (ORDER == 2) {
        return a.c0 * c + a.cx[0] * (xp[0] + xm[0]) + a.cy[0] * (yp[0] + ym[0]) + a.cz[0] * (zp[0] + zm[0]);
    } else {
        return lap_point<T, ORDER>(c, xm, xp, ym, yp, zm, zp, a);
    }
}

constexpr int kBarBytes = 1024;  // mbarriers + control words at the front of dynamic shared memory
constexpr int kMaxThreads = 448;
constexpr int kMaxConsumers = 416;
constexpr int kMaxThreadsKp = 352;  // complex states keep two register windows per thread
constexpr int kMaxConsumersKp = 320;
constexpr int kMaxStages = 16;

template <int ORDER>
constexpr int radius() { return ORDER == 2 ? 1 : (ORDER == 8 ? 4 : 3); }

struct WorkGrid {
    int tiles;   // y tiles of ty rows
    int nslab;   // z slabs
    int zslab;   // planes per slab
    int items;   // ns * tiles * nslab
};

// Persistent kernel: block b processes work items b, b + gridDim.x, ... where
// item = (state, y tile, z slab). The plane ring and its phases run on across
// items, so the producer streams the next item's planes while the consumers
// finish the current one. NC = 2 carries complex k-point states: a stage holds
// the real and the imaginary rows of one plane, and each point adds the
// first-derivative coupling -(1/2) 2i g.grad between the two parts
// (LaplasianKpoint8th_halo_f, GridDifferenceKpoint8th.h:18-122).
// NXC > 0: the row length nx as a compile-time constant (instantiated for the common
// grids), so that the y-neighbour offsets +-d*nx become immediate offsets of the
// shared-memory loads instead of per-load address arithmetic.
template <typename T, int ORDER, int PX, int NC, int NXC>
__global__ void __launch_bounds__(NC == 1 ? kMaxThreads : kMaxThreadsKp, 1)
    k_stencil_tma(const HamArgs<T> a, const WorkGrid wg, int nst) {
    constexpr int R = radius<ORDER>();
    constexpr int Q = 2 * R + 1;
    constexpr int NV = (R + PX - 1) / PX;  // neighbour vectors each side in x
    using VT = typename VecOf<T, PX>::type;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);               // [nst]
    uint64_t* empty = full + nst;                                      // [nst]
    volatile int* ctl = reinterpret_cast<volatile int*>(empty + nst);  // [0] abort, [1] last position issued
    T* ring = reinterpret_cast<T*>(smem + kBarBytes);

    const int nx = NXC > 0 ? NXC : a.nx, ny = a.ny, nz = a.nz, ty = a.ty;
    const int rows = ty + 2 * R;
    const int comp_elems = rows * nx;  // one part (real or imaginary) of a plane
    const int stage_elems = NC * comp_elems;
    const uint32_t stage_bytes = (uint32_t)stage_elems * sizeof(T);
    const int tpr = nx / PX;
    const int ncons = tpr * ty;
    const int ncons_warps = (ncons + 31) / 32;
    const int t = threadIdx.x;
    const long long plane = (long long)nx * ny;

    if (t == 0) {
        for (int i = 0; i < nst; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], (uint32_t)ncons_warps);
        }
        ctl[0] = 0;
        ctl[1] = -1;
        fence_mbar_init();
    }
    __syncthreads();

    if (t < 32) {
        // ---------------- producer warp: lane 0 streams planes ----------------
        if (t == 0 && !a.stall) {
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
                    T* dst = ring + (size_t)j * stage_elems;
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
                    ctl[1] = pos;
                }
            }
        }
    } else if (t < 32 + ncons) {
        // ---------------- consumer warps ----------------
        const unsigned wmask = __activemask();
        const int lane = t & 31;
        const int c = t - 32;
        const int ix0 = (c % tpr) * PX;
        const int ly = c / tpr;
        // shared-memory offsets inside a stage (constant for the thread)
        const int rowoff = (R + ly) * nx;
        int xoff[2 * NV];
#pragma unroll
        for (int v = 0; v < 2 * NV; ++v) {
            const int dv = (v < NV) ? (v - NV) : (v - NV + 1);
            int xx = ix0 + dv * PX;
            xx += (xx < 0) ? nx : 0;
            xx -= (xx >= nx) ? nx : 0;
            xoff[v] = rowoff + xx;
        }
        int pos = 0;  // ring position of the current item's first plane
        bool bad = false;
        for (int item = blockIdx.x; item < wg.items && !bad; item += gridDim.x) {
            const int slab = item % wg.nslab;
            const int tile = (item / wg.nslab) % wg.tiles;
            const int s = item / (wg.nslab * wg.tiles);
            const int iy = tile * ty + ly;
            const int zs = slab * wg.zslab;
            const int ze = min(nz, zs + wg.zslab);
            const long long col = (long long)iy * nx + ix0;

            // Register windows addressed by (step mod Q): the z-march is unrolled Q
            // times, so plane z - R + d sits in slot (k + d) % Q at unrolled step k and
            // the windows rotate by renaming instead of register moves (measured 3-13 %
            // faster for orders 4-8 and complex states; the 3-point order-2 window
            // keeps one step per iteration and shifts, which measured faster there).
            // q holds planes z-R .. z+R of the state, vq the potential of planes z .. z+R.
            constexpr bool kRot = !(ORDER == 2 && NC == 1);
            constexpr int KU = kRot ? Q : 1;
            auto sl = [](int k, int d) { return kRot ? (k + d) % Q : d; };
            Vec<T, PX> q[NC][Q];
            Vec<T, PX> vq[Q];
            // prologue: own z-window from the item's first 2R planes
            int j = pos % nst;
            uint32_t ph = (uint32_t)(pos / nst) & 1u;
            bool w = true;
#pragma unroll
            for (int d = 0; d < 2 * R; ++d) {
                if (w && !mbar_wait(&full[j], ph)) w = false;
#pragma unroll
                for (int cc = 0; cc < NC; ++cc)
                    q[cc][d].v = *reinterpret_cast<const VT*>(ring + j * stage_elems + cc * comp_elems + rowoff + ix0);
                if (++j == nst) { j = 0; ph ^= 1u; }
            }
            const T* vp = a.V + (long long)zs * plane + col;  // no wrap: zslab >= 2R keeps zs + R - 1 < ze <= nz
#pragma unroll
            for (int d = 0; d < R; ++d) vq[d].v = *reinterpret_cast<const VT*>(vp + (long long)d * plane);
            vp += (long long)R * plane;
            if (__any_sync(wmask, !w || ctl[0] != 0)) {
                bad = true;
                break;
            }
            __syncwarp(wmask);
            int jz = pos % nst;  // stage of plane z (starts at plane zs - R, advanced below)
            if (lane == 0)
                for (int d = 0; d < R; ++d) {  // planes zs-R .. zs-1 are done
                    mbar_arrive(&empty[jz]);
                    if (++jz == nst) jz = 0;
                }
            if (lane != 0) jz = (pos + R) % nst;
            int jp = j;             // stage of plane z + R (= position pos + 2R)
            uint32_t php = ph;
            T* hxp = a.HX + state_offset(a, s, true) + (long long)zs * plane + col;
            // per-k-point coefficients of the k-point kinetic term
            HamArgs<T> ak = a;
            if (NC == 2 && a.kco) {
                const T* kc = a.kco + (long long)(s / a.nsk) * 13;
                ak.c0 = kc[0];
#pragma unroll
                for (int d = 0; d < 4; ++d) {
                    ak.dx[d] = kc[1 + d];
                    ak.dy[d] = kc[5 + d];
                    ak.dz[d] = kc[9 + d];
                }
            }
            for (int z = zs; z < ze && !bad;) {
#pragma unroll
            for (int k = 0; k < KU; ++k) {
                if (z >= ze) break;
                if (z + R < ze) vq[sl(k, R)].v = *reinterpret_cast<const VT*>(vp);
                vp += plane;
                const bool ok = mbar_wait(&full[jp], php);
                if (__any_sync(wmask, !ok || ctl[0] != 0)) {
                    bad = true;
                    break;
                }
                T lap[NC][PX], der[NC][PX];
#pragma unroll
                for (int cc = 0; cc < NC; ++cc) {
                    const T* pzs = ring + jz * stage_elems + cc * comp_elems;
                    const T* pps = ring + jp * stage_elems + cc * comp_elems;
                    q[cc][sl(k, 2 * R)].v = *reinterpret_cast<const VT*>(pps + rowoff + ix0);
                    T xv[(2 * NV + 1) * PX];
#pragma unroll
                    for (int v = 0; v < 2 * NV; ++v) {
                        Vec<T, PX> wv;
                        wv.v = *reinterpret_cast<const VT*>(pzs + xoff[v]);
                        const int slot = (v < NV) ? v : v + 1;
#pragma unroll
                        for (int e = 0; e < PX; ++e) xv[slot * PX + e] = wv.e[e];
                    }
#pragma unroll
                    for (int e = 0; e < PX; ++e) xv[NV * PX + e] = q[cc][sl(k, R)].e[e];
                    Vec<T, PX> ypv[R], ymv[R];
#pragma unroll
                    for (int d = 1; d <= R; ++d) {
                        ypv[d - 1].v = *reinterpret_cast<const VT*>(pzs + rowoff + ix0 + d * nx);
                        ymv[d - 1].v = *reinterpret_cast<const VT*>(pzs + rowoff + ix0 - d * nx);
                    }
#pragma unroll
                    for (int e = 0; e < PX; ++e) {
                        T xm[R], xp[R], ym[R], yp[R], zm[R], zp[R];
#pragma unroll
                        for (int d = 1; d <= R; ++d) {
                            xm[d - 1] = xv[NV * PX + e - d];
                            xp[d - 1] = xv[NV * PX + e + d];
                            ym[d - 1] = ymv[d - 1].e[e];
                            yp[d - 1] = ypv[d - 1].e[e];
                            zm[d - 1] = q[cc][sl(k, R - d)].e[e];
                            zp[d - 1] = q[cc][sl(k, R + d)].e[e];
                        }
                        if constexpr (NC == 2) {
                            lap[cc][e] = lap_point_k<T, ORDER>(q[cc][sl(k, R)].e[e], xm, xp, ym, yp, zm, zp, ak);
                            der[cc][e] = der_point<T, ORDER>(xm, xp, ym, yp, zm, zp, ak);
                        } else {
                            lap[cc][e] = lap_point<T, ORDER>(q[cc][sl(k, R)].e[e], xm, xp, ym, yp, zm, zp, ak);
                        }
                    }
                }
                __syncwarp(wmask);
                if (lane == 0) mbar_arrive(&empty[jz]);  // plane z is no longer read
                if constexpr (NC == 1) {
                    Vec<T, PX> out;
#pragma unroll
                    for (int e = 0; e < PX; ++e) out.e[e] = vq[sl(k, 0)].e[e] * q[0][sl(k, R)].e[e] + lap[0][e];
                    *reinterpret_cast<VT*>(hxp) = out.v;
                } else {
                    // re: V re + L re - D im;  im: V im + L im + D re
                    Vec<T, PX> ore, oim;
#pragma unroll
                    for (int e = 0; e < PX; ++e) {
                        ore.e[e] = (vq[sl(k, 0)].e[e] * q[0][sl(k, R)].e[e] + lap[0][e]) - der[1][e];
                        oim.e[e] = (vq[sl(k, 0)].e[e] * q[1][sl(k, R)].e[e] + lap[1][e]) + der[0][e];
                    }
                    *reinterpret_cast<VT*>(hxp) = ore.v;
                    *reinterpret_cast<VT*>(hxp + a.hxim) = oim.v;
                }
                hxp += plane;
                if constexpr (!kRot) {
#pragma unroll
                    for (int cc = 0; cc < NC; ++cc)
#pragma unroll
                        for (int d = 0; d < 2 * R; ++d) q[cc][d] = q[cc][d + 1];
#pragma unroll
                    for (int d = 0; d < R; ++d) vq[d] = vq[d + 1];
                }
                ++z;
                if (++jz == nst) jz = 0;
                if (++jp == nst) { jp = 0; php ^= 1u; }
            }
            }
            if (bad) break;
            __syncwarp(wmask);
            if (lane == 0)
                for (int d = 0; d < R; ++d) {  // planes ze .. ze+R-1
                    mbar_arrive(&empty[jz]);
                    if (++jz == nst) jz = 0;
                }
            pos += ze - zs + 2 * R;
        }
        if (bad) {
            ctl[0] = 1;
            if (lane == 0) atomicExch(a.err, (int)QG_ERR_TIMEOUT);
        }
    }
    __syncthreads();
    if (t == 0 && ctl[0]) {
        // wind down: wait (bounded) for the fills still in flight
        const int last = ctl[1];
        for (int ps = max(0, last - nst + 1); ps <= last; ++ps) mbar_wait(&full[ps % nst], (uint32_t)(ps / nst) & 1u);
    }
}

// Rows per tile: the largest divisor of ny (<= 16) keeping the consumer threads within the kernel's limit.
template <typename T>
int tma_tile_rows(const HamArgs<T>& a, int nc, int order) {
    constexpr int PX = 16 / sizeof(T);
    // order 2 (3-plane window, DRAM-bound) measured fastest with at most 384 consumers
    const int maxc = nc == 1 ? (order == 2 ? 384 : kMaxConsumers) : kMaxConsumersKp;
    int ty = 0;
    for (int t = 1; t <= 16; ++t)
        if (a.ny % t == 0 && (a.nx / PX) * t <= maxc) ty = t;
    return ty;
}

// Ring stages that fit the shared-memory budget.
int ring_stages_for(int R, size_t stage_bytes) {
    const size_t budget = 200 * 1024 - kBarBytes;
    int nst = (int)std::min<size_t>(kMaxStages, budget / stage_bytes);
    const int need = std::max(2 * R, R + 2);
    return nst >= need ? nst : -1;
}

}  // namespace

// SM count of the current device, looked up once per device (devices of one process
// may differ: MIG slices, mixed parts). Racing first lookups store the same value.
int sm_count() {
    constexpr int kMaxDev = 64;
    static std::atomic<int> cache[kMaxDev];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= kMaxDev) dev = 0;
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n > 0) return n;
    int c = 0;
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    n = c > 0 ? c : 148;
    cache[dev].store(n, std::memory_order_relaxed);
    return n;
}

namespace {

template <typename T, int ORDER, int NC, int NXC = 0>
int launch_order(const HamArgs<T>& a, cudaStream_t st) {
    constexpr int PX = 16 / sizeof(T);
    constexpr int R = radius<ORDER>();
    if constexpr (NXC == 0 && ORDER >= 4) {
        // orders 4-8, FP64 and FP32: row lengths of the common grids compiled in
        switch (a.nx) {
            case 40: return launch_order<T, ORDER, NC, 40>(a, st);
            case 80: return launch_order<T, ORDER, NC, 80>(a, st);
            case 120: return launch_order<T, ORDER, NC, 120>(a, st);
            default: break;
        }
    }
    const size_t stage = (size_t)NC * (a.ty + 2 * R) * a.nx * sizeof(T);
    const int nst = ring_stages_for(R, stage);
    if (nst < 0) return QG_ERR_UNSUPPORTED;
    const size_t smem = kBarBytes + (size_t)nst * stage;
    auto kern = k_stencil_tma<T, ORDER, PX, NC, NXC>;
    if (allow_max_dynamic_smem(kern) != cudaSuccess)
        return QG_ERR_UNSUPPORTED;
    const int ncons = (a.nx / PX) * a.ty;
    const int threads = 32 + ncons;
    if (threads > (NC == 1 ? kMaxThreads : kMaxThreadsKp)) return QG_ERR_UNSUPPORTED;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1)
        return QG_ERR_UNSUPPORTED;
    const int G0 = sm_count() * per_sm;
    WorkGrid wg;
    wg.tiles = a.ny / a.ty;
    // z slabs: enough items for about four per block, slabs of at least 2R planes
    const long long base = (long long)a.ns * wg.tiles;
    wg.nslab = 1;
    while (base * wg.nslab < 4LL * G0 && a.nz / (wg.nslab * 2) >= 2 * R) wg.nslab *= 2;
    wg.zslab = (a.nz + wg.nslab - 1) / wg.nslab;
    wg.nslab = (a.nz + wg.zslab - 1) / wg.zslab;
    wg.items = (int)(base * wg.nslab);
    const int G = std::min(G0, wg.items);
    kern<<<G, threads, smem, st>>>(a, wg, nst);
    return QG_OK;
}

}  // namespace

template <typename T>
bool stencil_tma_ok(const HamArgs<T>& a, int order, int nc) {
    constexpr int PX = 16 / sizeof(T);
    const int R = order == 2 ? 1 : (order == 8 ? 4 : 3);
    if (nc != 1 && nc != 2) return false;
    if (nc == 2 && ((order != 2 && order != 6 && order != 8) || (a.xim % PX) || (a.hxim % PX))) return false;
    if (a.row) return false;  // the nonlocal scatter runs in k_scatter_all on this path
    if (a.nx % PX != 0 || ((uintptr_t)a.X % 16) || ((uintptr_t)a.HX % 16) || ((uintptr_t)a.V % 16) ||
        (a.ldx % PX) || (a.ldhx % PX) || !a.err || a.ny < 2 * R || a.nx < 2 * R)
        return false;
    const int ty = tma_tile_rows(a, nc, order);
    if (ty == 0) return false;
    const size_t stage = (size_t)nc * (ty + 2 * R) * a.nx * sizeof(T);
    return ring_stages_for(R, stage) > 0;
}

// Returns QG_ERR_UNSUPPORTED (launching nothing) when the shape or alignment
// does not fit this kernel; the caller then uses the register-window kernel.
template <typename T>
int launch_stencil_tma(const HamArgs<T>& a, int order, cudaStream_t st, int nc) {
    if (!stencil_tma_ok<T>(a, order, nc)) return QG_ERR_UNSUPPORTED;
    HamArgs<T> b = a;
    b.ty = tma_tile_rows(a, nc, order);
    if (nc == 2) {
        switch (order) {
            case 2: return launch_order<T, 2, 2>(b, st);
            case 6: return launch_order<T, 6, 2>(b, st);
            default: return launch_order<T, 8, 2>(b, st);
        }
    }
    switch (order) {
        case 2: return launch_order<T, 2, 1>(b, st);
        case 4: return launch_order<T, 4, 1>(b, st);
        case 6: return launch_order<T, 6, 1>(b, st);
        case 8: return launch_order<T, 8, 1>(b, st);
        default: return QG_ERR_INVALID;
    }
}

template bool stencil_tma_ok<double>(const HamArgs<double>&, int, int);
template bool stencil_tma_ok<float>(const HamArgs<float>&, int, int);
template int launch_stencil_tma<double>(const HamArgs<double>&, int, cudaStream_t, int);
template int launch_stencil_tma<float>(const HamArgs<float>&, int, cudaStream_t, int);

}  // namespace qg
