// Fused persistent delay-and-sum kernel with voxel blocking along the
// transmit-steering axis (sm_100a, EXACT tables, rectilinear grids).
//
// Why: a warp-wide 16-byte shared-memory load is served per quarter warp,
// i.e. it costs 4 L1 wavefronts whatever the addresses, so a thread that
// owns one voxel feeds only 4 FMAs per 16 bytes loaded and the kernel cannot
// pass ~25-30% of the FP32 pipe.  Here each thread owns VB = 4 voxels that
// differ only in v (the transmit-steering coordinate): they share the
// receive delay, apodisation and receive phasor, and their transmit delays
// differ by less than D samples over the block (checked on the host for
// the whole acquisition).  Per (tx, rx) step the thread loads the
// TAPS + D sample rows that cover all four voxels once and applies each
// voxel's weights shifted to its own first row (zeros elsewhere): one
// 16-byte load (two frames) feeds 16 FMAs.
//
// Tile: tu (receive axis) x tv*VB (steering axis) x tz (depth) voxels,
// 128 threads; windows staged as FP32 rows of a compile-time stride
// (FB * 8 + 16 bytes, so the loads use immediate offsets and 8 consecutive
// rows hit distinct banks): cp.async for complex64 slabs, register staging
// with one conversion for FP16/BF16 slabs.  Rows of the window past the end
// of the record are zero-filled, so no load needs clamping.  The
// interpolation weights come from polynomials (weight_poly.h; degree 8 for
// complex64 slabs, degree 6 for FP16 / BF16 slabs, whose ~5e-4 relative
// sample rounding is well above the degree-6 weight error of <= 8e-5), each
// mirrored pair of taps from one even and one odd chain.
//
// TM variant: the 2 x VB x FB accumulator words of a thread (128 at FB = 16,
// half the register file a thread can have) live in tensor memory instead
// of registers.  Per frame pair the warp loads the 16 words of the pair
// (VB voxels x 2 frames x re/im) from its own TMEM lanes, adds the step's
// terms and stores them back; a thread then fits in 128 registers instead of
// 255 (with spills), so four CTAs share an SM (16 warps instead of 8, all 512
// TMEM columns at FB = 16) to hide the shared-memory and FMA latencies.  TMEM loads and stores are warp-collective, so
// the accumulation runs for the whole warp whenever one of its lanes has a
// contribution; lanes without one read R rows of zeros kept in shared memory
// with zero weights, so they add exact zeros.
#pragma once

#include "das_common.cuh"
#include "poly_weights.cuh"
#include "tmem.cuh"

namespace rcabf {

constexpr int VB = VB_BLOCK;
constexpr int VB_THREADS = VB_THREADS_HOST;

template <int FB, int BYTES> struct VbChunk;
template <int FB> struct VbChunk<FB, 16> { using T = uint4; };
template <int FB> struct VbChunk<FB, 8> { using T = uint2; };
template <int FB> struct VbChunk<FB, 4> { using T = uint32_t; };

__device__ __forceinline__ float2 packed16_to_f2(uint32_t b, int store)
{
    if (store == ST_F16) {
        __half2 h;
        memcpy(&h, &b, 4);
        return __half22float2(h);
    }
    return make_float2(__uint_as_float(b << 16), __uint_as_float(b & 0xffff0000u));
}

// Window of the tile for one step: rows [lo, lo + count) cover every tap of
// every voxel plus D rows of shift; the first `data` rows exist in the
// record (the rest are zero-filled).
struct VbWindow {
    int lo, count, data;
    bool skip, overflow;
};

// Table bounds one step's window is computed from; loaded a step before
// they are needed, so the window computation does not wait on L2.
struct VbRanges {
    float2 rr, tr;   // receive / transmit table delay range of the tile
    float ab;        // aberration delay of the step
};

// step s = tx * n_ele + rx
__device__ __forceinline__ VbRanges vb_ranges(const FusedJob &J, int s, int n_steps, int tx, int rx, int tu, int tv,
                                              int tz)
{
    VbRanges r;
    if (s >= n_steps) {   // past the last step: an empty range (skipped)
        r.rr = make_float2(1.0f, 0.0f); r.tr = r.rr; r.ab = 0.0f;
        return r;
    }
    r.rr = J.rx_range[((int64_t)rx * J.tiles_u + tu) * J.tiles_z + tz];
    r.tr = J.tx_range[((int64_t)tx * J.tiles_v + tv) * J.tiles_z + tz];
    r.ab = ab_value(J.g, tx, rx);
    return r;
}

template <int KIND, int D>
__device__ __forceinline__ VbWindow vb_window(const FusedJob &J, const VbRanges &r, int wmax)
{
    using KT = KindTraits<KIND>;
    VbWindow w;
    w.lo = 0; w.count = 0; w.data = 0; w.overflow = false; w.skip = true;
    const float2 rr = r.rr, tr = r.tr;
    if (!(rr.x <= rr.y) || !(tr.x <= tr.y)) return w;
    float lo_f = __fadd_rn(__fadd_rn(tr.x, rr.x), r.ab);
    float hi_f = __fadd_rn(__fadd_rn(tr.y, rr.y), r.ab);
    const float fmax_n = (float)(J.n_sample);
    lo_f = fminf(fmaxf(floorf(lo_f), -1.0f), fmax_n);
    hi_f = fminf(fmaxf(floorf(hi_f), -1.0f), fmax_n);
    int lo = (int)lo_f - KT::LO;
    const int hi_taps = (int)hi_f - KT::LO + KT::TAPS - 1;   // last tap row any voxel uses
    lo = max(lo, 0);
    if (min(hi_taps, J.n_sample - 2) < lo) return w;         // no usable sample in the window
    const int hi = min(hi_taps, J.n_sample - 2) + D;         // + shift rows
    w.skip = false;
    w.lo = lo;
    w.count = hi - lo + 1;
    w.data = min(hi, J.n_sample - 1) - lo + 1;
    w.overflow = w.count > wmax;
    return w;
}

// Weights of each voxel shifted to its first row within the block's rows
// (zeros elsewhere) and its complex factor P = apod * exp(j phase_tx) *
// exp(j phase_rx) * exp(j phase_ab), zero for a voxel without a contribution
// (its weights then multiply finite staged rows into an exact zero).
template <int KIND, int D, int DEG>
__device__ __forceinline__ void vb_terms(const FusedParams &prm, const float (&fl)[VB], const float (&dd)[VB],
                                         bool (&ok)[VB], float base, const float (&txr)[VB],
                                         const float (&txq)[VB], float4 e, float2 abp,
                                         float (&ws)[VB][KindTraits<KIND>::TAPS + D], float2 (&P)[VB])
{
    constexpr int TAPS = KindTraits<KIND>::TAPS;
    constexpr int R = TAPS + D;
#pragma unroll
    for (int v = 0; v < VB; ++v) {
        int o = (int)(fl[v] - base);
        if (ok[v] && o > D) { atomicAdd(prm.err_count, 1ull); ok[v] = false; }
        o = ok[v] ? o : 0;
        float w[TAPS];
        poly_weights<KIND, DEG>(ok[v] ? dd[v] : 0.0f, w);   // finite whatever the index of a masked voxel
#pragma unroll
        for (int k = 0; k < R; ++k) {
            float a = (k < TAPS) ? w[k] : 0.0f;
            if constexpr (D >= 1) { if (o == 1) a = (k >= 1 && k - 1 < TAPS) ? w[k - 1] : 0.0f; }
            if constexpr (D >= 2) { if (o == 2) a = (k >= 2 && k - 2 < TAPS) ? w[k - 2] : 0.0f; }
            ws[v][k] = a;   // finite; a voxel without a contribution has P = 0
        }
        const float qx = fmaf(txr[v], e.y, -txq[v] * e.z), qy = fmaf(txr[v], e.z, txq[v] * e.y);
        P[v] = ok[v] ? make_float2(fmaf(qx, abp.x, -qy * abp.y), fmaf(qx, abp.y, qy * abp.x))
                     : make_float2(0.f, 0.f);
    }
}

// Weighted row sums of one frame pair for every voxel: lo[v] = sum_k
// ws[v][k] * (word 0, word 1) of row k, hi[v] = the same of (word 2, word
// 3), two FP32 FMAs per instruction (fma.rn.f32x2, the same IEEE operation
// on each half as fmaf).  Rows hold a frame pair as (re0, im0, re1, im1)
// when staged by cp.async (complex64 slabs) and as (re0, re1, im0, im1)
// when staged from registers (FP16/BF16 slabs): see VbPlanar.
template <int R, int STRIDE>
__device__ __forceinline__ void vb_pair_sums(const char *rows, const float (&ws)[VB][R], float2 (&lo)[VB],
                                             float2 (&hi)[VB])
{
#pragma unroll
    for (int v = 0; v < VB; ++v) { lo[v] = make_float2(0.f, 0.f); hi[v] = make_float2(0.f, 0.f); }
#pragma unroll
    for (int k = 0; k < R; ++k) {
        const float4 x = *reinterpret_cast<const float4 *>(rows + k * STRIDE);
        const float2 xl = make_float2(x.x, x.y), xh = make_float2(x.z, x.w);
#pragma unroll
        for (int v = 0; v < VB; ++v) {
            const float2 w2 = make_float2(ws[v][k], ws[v][k]);
            lo[v] = __ffma2_rn(w2, xl, lo[v]);
            hi[v] = __ffma2_rn(w2, xh, hi[v]);
        }
    }
}

// Staged frame-pair layout: planar (re0, re1, im0, im1) for register
// staging, where the conversion writes the words in any order, so that the
// phasor products of both frames pair up (re with re, im with im) for
// fma.rn.f32x2; interleaved (re0, im0, re1, im1) for cp.async staging,
// which copies complex64 slabs as they are.
template <int STORE> struct VbPlanar { static constexpr bool value = STORE != ST_F32; };

// Degree of the weight polynomials per slab storage: 8 for complex64
// (weight error ~5e-7), 6 for FP16 / BF16 (weight error <= 8e-5, below the
// ~5e-4 relative rounding of the stored samples).
template <int STORE> struct VbWeightDeg { static constexpr int value = STORE == ST_F32 ? 8 : 6; };

// (re, im) of frames 2p, 2p + 1 from a pair's four words in the layout
template <bool PL>
__device__ __forceinline__ void vb_unpack(float w0, float w1, float w2, float w3, float2 &f0, float2 &f1)
{
    if constexpr (PL) { f0 = make_float2(w0, w2); f1 = make_float2(w1, w3); }
    else { f0 = make_float2(w0, w1); f1 = make_float2(w2, w3); }
}

template <int KIND, int FB, int STORE, int D, bool TM>
__global__ void __launch_bounds__(VB_THREADS, TM ? VB_TM_MIN_BLOCKS : VB_MIN_BLOCKS)
fused_vb_kernel(const __grid_constant__ FusedParams prm)
{
    static_assert(FB % 2 == 0, "frames are processed in pairs");
    static_assert(!TM || VB == 4, "a TMEM access moves the 16 words of VB = 4 voxels x one frame pair");
    using T = typename StoreT<STORE>::T;
    using KT = KindTraits<KIND>;
    constexpr int TAPS = KT::TAPS;
    constexpr int R = TAPS + D;                        // rows a thread reads per step
    constexpr bool ASYNC = (STORE == ST_F32);
    constexpr bool PL = VbPlanar<STORE>::value;        // staged frame-pair layout
    constexpr int NST = ASYNC ? 3 : 2;
    constexpr int ES = (int)sizeof(T);
    constexpr int RAWB = FB * ES;
    constexpr int SROWB = FB * 8;
    constexpr int STRIDE = SROWB + 16;                 // staged row stride (bytes)
    constexpr int CS = RAWB < 16 ? RAWB : 16;
    constexpr int CPR = RAWB / CS;
    constexpr int SREGS = VB_STAGE_REGS;               // staging chunks per thread
    using Chunk = typename VbChunk<FB, CS>::T;

    extern __shared__ __align__(16) unsigned char smem[];
    const int tid = threadIdx.x;
    const int stage_bytes = prm.wmax * STRIDE;
    {
        unsigned dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        // (TM: R rows of zeros follow the stages)
        if (dyn < (unsigned)(NST * stage_bytes + (TM ? R * STRIDE : 0)) || prm.row_words * 4 != STRIDE ||
            (!ASYNC && prm.wmax * CPR > SREGS * VB_THREADS)) {
            if (tid == 0) atomicAdd(prm.err_count, 1ull);
            return;
        }
    }
    unsigned char *stages = smem;

    // TM: warp 0 allocates the CTA's columns; each warp addresses the 32
    // lanes of its quadrant, each thread its own lane
    constexpr uint32_t TCOLS = (uint32_t)vb_tmem_cols_host(FB);
    uint32_t tlane = 0;
    const int zero_off = NST * stage_bytes;   // TM: offset of R staged rows of zeros
    if constexpr (TM) {
        __shared__ uint32_t tbase;
        for (int i = tid; i < R * STRIDE / 16; i += VB_THREADS)
            *reinterpret_cast<float4 *>(smem + zero_off + 16 * i) = make_float4(0.f, 0.f, 0.f, 0.f);
        if (tid < 32) {
            tmem_alloc(&tbase, TCOLS);
            tmem_relinquish();
        }
        tmem_fence_before_sync();
        __syncthreads();
        tmem_fence_after_sync();
        tlane = tbase + ((uint32_t)(32 * ((tid >> 5) & 3)) << 16);
    }

    for (int64_t item = blockIdx.x; item < prm.n_items; item += gridDim.x) {
        int ji = 0;
        while (ji + 1 < prm.n_jobs && prm.jobs[ji + 1].item_begin <= item) ++ji;
        const FusedJob &J = prm.jobs[ji];
        const DevGeom &g = J.g;
        const int lu = tid % J.tu;
        const int lvb = (tid / J.tu) % J.tv;
        const int lz = tid / (J.tu * J.tv);
        const int64_t local = item - J.item_begin;
        const int64_t n_tiles = (int64_t)J.tiles_z * J.tiles_u * J.tiles_v;
        const int fb = (int)(local / n_tiles);
        const int64_t tile = local % n_tiles;
        const int tz = (int)(tile % J.tiles_z);
        const int tu = (int)((tile / J.tiles_z) % J.tiles_u);
        const int tv = (int)(tile / ((int64_t)J.tiles_z * J.tiles_u));
        const int64_t iz = (int64_t)tz * J.tz + lz;
        const int64_t iu = (int64_t)tu * J.tu + lu;
        const int64_t iv0 = ((int64_t)tv * J.tv + lvb) * VB;
        const bool zu = iz < g.n_z && iu < g.n_u;
        const int64_t rem = g.n_v - iv0;
        const int nvv = !zu ? 0 : rem <= 0 ? 0 : rem >= VB ? VB : (int)rem;
        const int64_t rxkey = iu * g.n_z + iz;
        const int64_t n_rxkey = g.n_u * g.n_z;
        const int64_t n_txkey = g.n_v * g.n_z;
        const int n_steps = g.n_tx * g.n_ele;
        const char *S = reinterpret_cast<const char *>(J.S);

        float2 acc[VB][FB];
#pragma unroll
        for (int v = 0; v < VB; ++v)
#pragma unroll
            for (int f = 0; f < FB; ++f) acc[v][f] = make_float2(0.f, 0.f);
        // TM: words [16 p, 16 p + 16) of a lane hold frames 2p, 2p + 1 of
        // its voxels: voxel v at 4 v + the staged layout (VbPlanar: re 2p,
        // re 2p+1, im 2p, im 2p+1; else re 2p, im 2p, re 2p+1, im 2p+1)
        auto tm_zero = [&]() {
            uint32_t z[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) z[i] = 0u;
            __syncwarp();   // TMEM accesses are warp-collective: converge first
#pragma unroll
            for (int c = 0; c < FB; c += 2) tmem_st16(tlane + (uint32_t)(c * 8), z);
        };
        // per-voxel, per-frame output of the accumulators (TM: read back
        // from the lane's words), optionally added to what `out` holds
        auto emit = [&](int64_t frame_stride, int64_t frame_off) {
#pragma unroll
            for (int c = 0; c < FB; c += 2) {
                float2 a[VB][2];
                if constexpr (TM) {
                    uint32_t w[16];
                    __syncwarp();
                    tmem_wait_st();
                    tmem_ld16(tlane + (uint32_t)(c * 8), w);
                    tmem_wait_ld16(w);
#pragma unroll
                    for (int v = 0; v < VB; ++v)
                        vb_unpack<PL>(__uint_as_float(w[4 * v]), __uint_as_float(w[4 * v + 1]),
                                      __uint_as_float(w[4 * v + 2]), __uint_as_float(w[4 * v + 3]), a[v][0], a[v][1]);
                } else {
#pragma unroll
                    for (int v = 0; v < VB; ++v) { a[v][0] = acc[v][c]; a[v][1] = acc[v][c + 1]; }
                }
#pragma unroll
                for (int v = 0; v < VB; ++v) {
                    if (v < nvv) {
                        const int64_t pix = iz * g.s_z + iu * g.s_u + (iv0 + v) * g.s_v;
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            const int fr = fb * FB + c + h;
                            if (fr < J.n_frame) {
                                float2 *o = J.out + (int64_t)fr * frame_stride + frame_off + pix;
                                if (J.accumulate) { float2 q = *o; q.x += a[v][h].x; q.y += a[v][h].y; *o = q; }
                                else *o = a[v][h];
                            }
                        }
                    }
                }
            }
        };
        if constexpr (TM) tm_zero();

        // Transmit order rotated per tile: a hash of the tile picks the
        // quarter of the transmits the item starts from, so CTAs that share
        // an SM run their per-step setup and their frame-pair FMAs out of
        // phase rather than in lock step (started together, with equal step
        // costs, they would stay aligned).  Whole transmits: per-transmit
        // outputs stay complete.  The loop counter s stays the step's
        // position in the item; eff(s) is the acquisition step it works on.
        const int tx0 = g.n_tx >= 4 ? (int)((((uint32_t)tile * 0x9E3779B1u) >> 30) * (uint32_t)g.n_tx / 4u) : 0;
        const int s0 = tx0 * g.n_ele;
        auto eff = [&](int s) { const int e = s + s0; return e < n_steps ? e : e - n_steps; };
        // slabs are ordered by step tx * n_ele + rx, then frame block
        auto slab = [&](int s) -> const char * { return S + ((int64_t)eff(s) * J.n_fb + fb) * J.slab_bytes; };
        // (tx, rx) of step s: divided once per item, then advanced per step
        auto advance = [&](int &tx, int &rx) {
            if (++rx == g.n_ele) {
                rx = 0;
                if (++tx == g.n_tx) tx = 0;
            }
        };
        auto window = [&](int s) -> VbWindow {
            VbWindow w;
            w.skip = true; w.lo = 0; w.count = 0; w.data = 0; w.overflow = false;
            if (s >= n_steps) return w;
            return vb_window<KIND, D>(J, vb_ranges(J, s, n_steps, eff(s) / g.n_ele, eff(s) % g.n_ele, tu, tv, tz),
                                      prm.wmax);
        };
        // rows [data, count) of a staged buffer hold zeros (shift rows past the record)
        auto zero_tail = [&](unsigned char *dst, const VbWindow &w) {
            const int nz = (w.count - w.data) * (SROWB / 16);
            for (int c = tid; c < nz; c += VB_THREADS) {
                const int r = w.data + c / (SROWB / 16), q = c % (SROWB / 16);
                *reinterpret_cast<float4 *>(dst + r * STRIDE + q * 16) = make_float4(0.f, 0.f, 0.f, 0.f);
            }
        };
        auto issue_async = [&](int s, const VbWindow &w) {
            if (!w.skip && !w.overflow) {
                const char *src = slab(s) + (int64_t)w.lo * RAWB;
                unsigned char *dst = stages + (s % NST) * stage_bytes;
                const int nch = w.data * CPR;
                for (int c = tid; c < nch; c += VB_THREADS) {
                    const int r = c / CPR, q = c % CPR;
                    cp_async<CS>(dst + r * STRIDE + q * CS, src + (int64_t)r * RAWB + q * CS);
                }
                zero_tail(dst, w);
            }
            cp_async_commit();
        };
        Chunk regs[SREGS];
        auto load_regs = [&](int s, const VbWindow &w) {
            if (w.skip || w.overflow) return;
            const char *src = slab(s) + (int64_t)w.lo * RAWB;
            const int nch = w.data * CPR;
#pragma unroll
            for (int k = 0; k < SREGS; ++k) {
                const int c = tid + k * VB_THREADS;
                if (c < nch) regs[k] = __ldg(reinterpret_cast<const Chunk *>(src + (int64_t)c * CS));
            }
        };
        auto store_regs = [&](int s, const VbWindow &w) {
            if (w.skip || w.overflow) return;
            unsigned char *dst = stages + (s % NST) * stage_bytes;
            const int nch = w.data * CPR;
#pragma unroll
            for (int k = 0; k < SREGS; ++k) {
                const int c = tid + k * VB_THREADS;
                if (c < nch) {
                    const int r = c / CPR, q = c % CPR;
                    float2 *o = reinterpret_cast<float2 *>(dst + r * STRIDE + q * CS * 2);
                    uint32_t b[CS / 4];
                    memcpy(b, &regs[k], CS);
#pragma unroll
                    for (int v = 0; v < CS / 4; v += 2) {
                        if (v + 1 < CS / 4) {
                            const float2 x0 = packed16_to_f2(b[v], STORE), x1 = packed16_to_f2(b[v + 1], STORE);
                            // planar frame pair (re0, re1, im0, im1), VbPlanar
                            *reinterpret_cast<float4 *>(o + v) = make_float4(x0.x, x1.x, x0.y, x1.y);
                        } else {
                            o[v] = packed16_to_f2(b[v], STORE);
                        }
                    }
                }
            }
            zero_tail(dst, w);
        };

        VbWindow wA = window(0), wB = window(1), wC;
        int tx3 = eff(2 % n_steps) / g.n_ele, rx3 = eff(2 % n_steps) % g.n_ele;   // step of the ranges loaded next
        VbRanges rnext = vb_ranges(J, 2, n_steps, tx3, rx3, tu, tv, tz);   // ranges of the step two ahead
        advance(tx3, rx3);
        if constexpr (ASYNC) {
            issue_async(0, wA);
            issue_async(1, wB);
        } else {
            load_regs(0, wA);
            store_regs(0, wA);
            load_regs(1, wB);
            __syncthreads();
        }

        // per-transmit state of the thread's voxels: index part, phasor, cone
        float txi[VB], txr[VB], txq[VB];
        unsigned cone_bits = 0;
#pragma unroll
        for (int v = 0; v < VB; ++v) { txi[v] = 0.f; txr[v] = 0.f; txq[v] = 0.f; }
        float4 enext = nvv > 0 ? __ldg(&g.rx_tab[rxkey]) : make_float4(0.f, 0.f, 0.f, 0.f);

        int tx = tx0, rx = 0;   // of step s
        for (int s = 0; s < n_steps; ++s, advance(tx, rx)) {
            if constexpr (ASYNC) {
                cp_async_wait<NST - 2>();
                __syncthreads();
                wC = vb_window<KIND, D>(J, rnext, prm.wmax);
                rnext = vb_ranges(J, s + 3, n_steps, tx3, rx3, tu, tv, tz);
                advance(tx3, rx3);
                issue_async(s + 2, wC);
            }
            const float4 e = enext;
            if (nvv > 0 && s + 1 < n_steps)
                enext = __ldg(&g.rx_tab[(int64_t)(rx + 1 == g.n_ele ? 0 : rx + 1) * n_rxkey + rxkey]);
            if (rx == 0 && nvv > 0) {
                const float4 *txrow = g.tx_tab + (int64_t)tx * n_txkey + iz;
                cone_bits = 0;
                const bool cu = g.cone_u == nullptr || g.cone_u[(int64_t)tx * n_rxkey + rxkey] != 0;
#pragma unroll
                for (int v = 0; v < VB; ++v) {
                    if (v < nvv) {
                        const float4 t = __ldg(&txrow[(iv0 + v) * g.n_z]);
                        txi[v] = t.x; txr[v] = t.y; txq[v] = t.z;
                        if (cu && t.w != 0.0f) cone_bits |= 1u << v;
                    }
                }
            }

            if constexpr (!TM) {
                if (!wA.skip && cone_bits != 0 && e.w > 0.0f) {
                    const float ab = ab_value(g, tx, rx);
                    const float2 abp = ab_phasor(g, tx, rx);
                    // sample index of each voxel; rows are shared from the lowest
                    float fl[VB], dd[VB];
                    bool ok[VB];
                    float base = 3.0e38f;
#pragma unroll
                    for (int v = 0; v < VB; ++v) {
                        const float idx = __fadd_rn(__fadd_rn(txi[v], e.x), ab);
                        fl[v] = floorf(idx);
                        dd[v] = idx - fl[v];
                        ok[v] = ((cone_bits >> v) & 1u) && fl[v] >= (float)KT::LO &&
                                fl[v] < (float)(J.n_sample - 1 - KT::HI);
                        if (ok[v]) base = fminf(base, fl[v]);
                    }
                    if (base < 2.0e38f) {
                        float ws[VB][R];
                        float2 P[VB];
                        vb_terms<KIND, D, VbWeightDeg<STORE>::value>(prm, fl, dd, ok, base, txr, txq, e, abp, ws, P);
                        const int row0 = (int)base - KT::LO - wA.lo;
                        if (row0 < 0 || row0 + R > wA.count || wA.overflow) {
                            atomicAdd(prm.err_count, 1ull);   // never expected: window bound violated
                        } else {
                            const char *rows = reinterpret_cast<const char *>(stages) +
                                               (s % NST) * stage_bytes + row0 * STRIDE;
#pragma unroll
                            for (int c = 0; c < FB; c += 2) {
                                float2 lo[VB], hi[VB];
                                vb_pair_sums<R, STRIDE>(rows + c * 8, ws, lo, hi);
#pragma unroll
                                for (int v = 0; v < VB; ++v) {
                                    float2 t0, t1;   // interpolated (re, im) of frames c, c + 1
                                    vb_unpack<PL>(lo[v].x, lo[v].y, hi[v].x, hi[v].y, t0, t1);
                                    float2 &a0 = acc[v][c], &a1 = acc[v][c + 1];
                                    a0.x = fmaf(P[v].x, t0.x, fmaf(-P[v].y, t0.y, a0.x));
                                    a0.y = fmaf(P[v].x, t0.y, fmaf(P[v].y, t0.x, a0.y));
                                    a1.x = fmaf(P[v].x, t1.x, fmaf(-P[v].y, t1.y, a1.x));
                                    a1.y = fmaf(P[v].x, t1.y, fmaf(P[v].y, t1.x, a1.y));
                                }
                            }
                        }
                    }
                }
            } else {
                // every lane computes its terms (lanes without voxels carry
                // zeros); the warp accumulates when any lane contributes
                const bool act = !wA.skip && cone_bits != 0 && e.w > 0.0f;
                const float ab = ab_value(g, tx, rx);
                const float2 abp = ab_phasor(g, tx, rx);
                float fl[VB], dd[VB];
                bool ok[VB];
                float base = 3.0e38f;
#pragma unroll
                for (int v = 0; v < VB; ++v) {
                    const float idx = __fadd_rn(__fadd_rn(txi[v], e.x), ab);
                    fl[v] = floorf(idx);
                    dd[v] = idx - fl[v];
                    ok[v] = act && ((cone_bits >> v) & 1u) && fl[v] >= (float)KT::LO &&
                            fl[v] < (float)(J.n_sample - 1 - KT::HI);
                    if (ok[v]) base = fminf(base, fl[v]);
                }
                bool use = base < 2.0e38f;
                int row0 = use ? (int)base - KT::LO - wA.lo : 0;
                if (use && (row0 < 0 || row0 + R > wA.count || wA.overflow)) {
                    atomicAdd(prm.err_count, 1ull);   // never expected: window bound violated
                    use = false;
                }
                if (!use) {   // all weights zero, rows of zeros: the lane adds exact zeros
#pragma unroll
                    for (int v = 0; v < VB; ++v) ok[v] = false;
                }
                if (__any_sync(0xffffffffu, use)) {
                    float ws[VB][R];
                    float2 P[VB];
                    vb_terms<KIND, D, VbWeightDeg<STORE>::value>(prm, fl, dd, ok, use ? base : 0.0f, txr, txq, e, abp, ws,
                                                                 P);
                    const char *rows = reinterpret_cast<const char *>(stages) +
                                       (use ? (s % NST) * stage_bytes + row0 * STRIDE : zero_off);
                    __syncwarp();     // converged after the divergent checks above
                    tmem_wait_st();   // the previous step's stores are visible to the loads below
                    // (one pair per iteration: unrolled by two the loop spills 56
                    // bytes at 128 registers and measured 0.6% slower, fully
                    // unrolled it measured 14% slower)
#pragma unroll 1
                    for (int c = 0; c < FB; c += 2) {
                        uint32_t w[16];
                        tmem_ld16(tlane + (uint32_t)(c * 8), w);
                        float2 lo[VB], hi[VB];
                        vb_pair_sums<R, STRIDE>(rows + c * 8, ws, lo, hi);
                        tmem_wait_ld16(w);
#pragma unroll
                        for (int v = 0; v < VB; ++v) {
                            if constexpr (PL) {
                                // words (re0, re1, im0, im1); lo = interpolated re of
                                // both frames, hi = im: re += Px re - Py im, im +=
                                // Px im + Py re, both frames per fma.rn.f32x2, in
                                // the scalar kernel's order
                                float2 re = make_float2(__uint_as_float(w[4 * v]), __uint_as_float(w[4 * v + 1]));
                                float2 im = make_float2(__uint_as_float(w[4 * v + 2]), __uint_as_float(w[4 * v + 3]));
                                const float2 px = make_float2(P[v].x, P[v].x), py = make_float2(P[v].y, P[v].y);
                                const float2 npy = make_float2(-P[v].y, -P[v].y);
                                re = __ffma2_rn(px, lo[v], __ffma2_rn(npy, hi[v], re));
                                im = __ffma2_rn(px, hi[v], __ffma2_rn(py, lo[v], im));
                                w[4 * v] = __float_as_uint(re.x);
                                w[4 * v + 1] = __float_as_uint(re.y);
                                w[4 * v + 2] = __float_as_uint(im.x);
                                w[4 * v + 3] = __float_as_uint(im.y);
                            } else {
                                const float a0x = __uint_as_float(w[4 * v]), a0y = __uint_as_float(w[4 * v + 1]);
                                const float a1x = __uint_as_float(w[4 * v + 2]), a1y = __uint_as_float(w[4 * v + 3]);
                                const float2 t0 = lo[v], t1 = hi[v];
                                w[4 * v] = __float_as_uint(fmaf(P[v].x, t0.x, fmaf(-P[v].y, t0.y, a0x)));
                                w[4 * v + 1] = __float_as_uint(fmaf(P[v].x, t0.y, fmaf(P[v].y, t0.x, a0y)));
                                w[4 * v + 2] = __float_as_uint(fmaf(P[v].x, t1.x, fmaf(-P[v].y, t1.y, a1x)));
                                w[4 * v + 3] = __float_as_uint(fmaf(P[v].x, t1.y, fmaf(P[v].y, t1.x, a1y)));
                            }
                        }
                        tmem_st16(tlane + (uint32_t)(c * 8), w);
                    }
                }
            }

            if (rx == g.n_ele - 1 && !J.compound) {   // per-transmit output
                emit((int64_t)g.n_tx * g.n_pix, (int64_t)tx * g.n_pix);
                if constexpr (TM) {
                    tm_zero();
                } else {
#pragma unroll
                    for (int v = 0; v < VB; ++v)
#pragma unroll
                        for (int f = 0; f < FB; ++f) acc[v][f] = make_float2(0.f, 0.f);
                }
            }

            if constexpr (!ASYNC) {
                store_regs(s + 1, wB);
                wC = vb_window<KIND, D>(J, rnext, prm.wmax);
                rnext = vb_ranges(J, s + 3, n_steps, tx3, rx3, tu, tv, tz);
                advance(tx3, rx3);
                load_regs(s + 2, wC);
                __syncthreads();
            }
            wA = wB;
            wB = wC;
        }
        if constexpr (ASYNC) cp_async_wait<0>();
        __syncthreads();

        if (J.compound) emit(g.n_pix, 0);
    }
    if constexpr (TM) {
        // every load was waited for; the last stores complete before the free
        __syncwarp();
        tmem_wait_st();
        tmem_fence_before_sync();
        __syncthreads();
        if (tid < 32) {
            tmem_fence_after_sync();
            tmem_dealloc(tlane, TCOLS);   // warp 0's lane address is the allocation's base
        }
    }
}

}  // namespace rcabf
