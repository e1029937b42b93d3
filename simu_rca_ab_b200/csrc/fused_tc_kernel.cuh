// Delay-and-sum on the tensor cores (sm_100a tcgen05.mma), EXACT tables,
// FP16 or BF16 slabs, rectilinear grids, transmits compounded.
//
// Formulation.  For a tile of 128 voxels (tu along the receive axis x tv
// along the steering axis, one depth; the planner picks the shape whose
// windows are shortest) and one (tx, rx) step, the sample
// rows every voxel of the tile touches form one window [lo, lo + K) of the
// step's slab, K <= 32 rows.  With W[m][k] = P_m w_m(k - o_m) (the voxel's
// interpolation weights placed at its own row offset o_m inside the window,
// times its complex factor P = apod * transmit phasor * receive phasor), the
// step's contribution to every frame f is a banded matrix product
//     out[m][f] += sum_k W[m][k] * S[lo + k][f],
// and summing over all (tx, rx) steps is one long contraction: the tile's
// accumulators stay in tensor memory across the whole acquisition.  S rows
// hold the frames of a block as (re, im) FP16 (BF16) pairs, and the ingest
// writes a second copy S' of the slabs holding (-im, re), so with the real and
// imaginary parts of W in two matrices one accumulator takes both:
//     D = Re(W) . S + Im(W) . S'    (N = 2 FB columns, (re, im) per frame)
// i.e. D[re] = Re(W) S_re - Im(W) S_im, D[im] = Re(W) S_im + Im(W) S_re.
// The accumulator holds N = 2 FB FP32 columns, up to 416 (frame blocks up to
// 208 frames; 232 with single FP16 weights): one MMA instruction covers at
// most N = 256, so wider blocks issue two per weight matrix (columns
// [0, 256) and [256, N), the second B operand starting at its fifth 64-element
// panel).  Frame blocks are as wide as the tensor memory allows because the
// weights are built once per (tile, step, frame block): the builders' work
// per frame falls as the block grows, while the MMA work per frame stays.
// Weights are formed in FP32 exactly as the SIMT kernels form them (degree-6
// polynomials, FP32 phasors) and enter the MMA in the slabs' type (A and B
// of one MMA have the same type): SPLIT = true adds a second term holding
// the remainder (hi + lo carries ~22 bits in FP16, ~16 in BF16; the MMA
// products are exact and summed in FP32), SPLIT = false keeps the single
// FP16 rounding (~11 bits; not offered for BF16).  All weights are scaled by
// 2^8 (undone in the epilogue) so that the remainder terms stay out of the
// FP16 subnormal range.
//
// Records.  A step's window is one or two 16-row chunks; each chunk is one
// record (one K = 16 slice of the contraction), so every record has the same
// shape: one weight slot of NMAT matrices of 8 tensor-memory columns, one
// window stage of 16 rows of S and of S'.
//
// Roles (480 threads; tiles in depth-slowest order): three groups of four
// warps build the weight
// matrices, one voxel per thread, straight into tensor memory (lane = voxel
// row; tcgen05.st), taking records in turn (group g the records q with
// q mod 3 = g, so that the groups' dependent setup chains overlap), and the
// group that
// meets an item's end record writes that item's outputs; warp 12, the
// producer, computes the windows of 32 steps at a time and each of its lanes
// with an active step writes that step's chunk records into a ring of TC_NSR
// record slots, at least TC_NPUB records ahead of the MMAs; warp 14, the
// loader, follows the ring one record at a time and loads each record's rows
// with 3-D TMA (128-byte swizzle) into its stage of a ring of TC_NSB
// shared-memory stages as soon as that stage is free, so that the loads run
// up to TC_NSB records ahead of the MMAs with no gap between rounds; warp 13
// issues the MMAs (A from one of TC_NSA tensor-memory weight slots, B from
// shared memory) and commits them to the stage's "empty" barrier, which also
// tells the builders the slot is free.
// Steps whose window is empty for the whole tile are skipped by every role
// alike: the producer passes each active chunk's record (step, window
// start, window chunks, chunk, item) through a ring of TC_NSR record slots
// -- the builders start on a record as soon as it is written, ahead of its
// rows' load -- then an end-of-item record (with the item's count of
// records), and after the last item one final record per builder group.
// Every wait
// is bounded (mbar_wait): a wait that runs out sets an abort flag, counts an
// error and every role leaves its loop.
//
// Tensor memory (512 columns, one CTA per SM): D at column 0 (N16 <= 416
// columns), then TC_NSA slots of NMAT weight matrices of 8 columns (16 FP16
// per row: K = 16).
#pragma once

#include <cuda.h>

#include <type_traits>

#include "das_common.cuh"
#include "poly_weights.cuh"
#include "tc_common.cuh"

namespace rcabf {

constexpr int TC_GROUPS = 3;               // builder groups of 4 warps
constexpr int TC_THREADS = 32 * (4 * TC_GROUPS + 3);
constexpr int TC_PRODUCER_WARP = 4 * TC_GROUPS, TC_MMA_WARP = 4 * TC_GROUPS + 1, TC_LOADER_WARP = 4 * TC_GROUPS + 2;
constexpr int TC_KCH = TC_MAX_ROWS / 16;   // 16-row chunks per step window at most (windows <= 32 rows)
constexpr int TC_NSA = 3;                  // weight-matrix slots in tensor memory: record q uses slot q mod TC_NSA
constexpr int TC_NSB = 6;                  // window stages in shared memory
static_assert(TC_NSB > TC_NSA, "slot reuse is signalled through the window stages");
constexpr int TC_NSR = 2 * TC_NSB;         // records in flight (a ring of its own, ahead of the window loads)
constexpr int TC_NPUB = TC_NSR / 2;        // records the producer writes per round
static_assert(TC_GROUPS <= TC_NPUB, "the final records are written in one round");
static_assert(TC_NSR >= TC_NSB, "a record is written before its window is loaded");
// A stage holds one 16-row chunk of S and the same rows of S'; a chunk is
// tc_panels(fb) 64-element panels of 16 rows x 128 bytes (2048 bytes each,
// 128-byte swizzle), loaded by one 3-D TMA (x = element in the panel,
// y = row, z = panel); the MMA's leading offset is the 2048-byte panel step.
constexpr int TC_PANEL_BYTES = 2048;
constexpr float TC_SCALE = 256.0f;
constexpr int TC_NMAX = 256;              // widest N of one MMA instruction (M = 128)
constexpr RCABF_HD int tc_nmat(bool split) { return split ? 4 : 2; }
constexpr RCABF_HD int tc_n16(int fb) { return (2 * fb + 15) / 16 * 16; }
constexpr RCABF_HD int tc_panels(int fb) { return (2 * fb + 63) / 64; }
// tensor-memory columns the kernel needs at frame block fb
constexpr RCABF_HD int tc_tmem_cols(int fb, bool split) { return tc_n16(fb) + TC_NSA * tc_nmat(split) * 8; }
// largest frame block (a multiple of 8): the accumulator and the weight
// slots share the 512 tensor-memory columns (208 frames with hi +
// remainder weights, 232 with single FP16 weights)
constexpr RCABF_HD int tc_max_fb(bool split) { return (512 - TC_NSA * tc_nmat(split) * 8) / 2 / 8 * 8; }
// dynamic shared memory: TC_NSB stages of B panels + 1 KB for the 1024-byte alignment
constexpr RCABF_HD size_t tc_smem_bytes(int fb) { return (size_t)TC_NSB * 2 * tc_panels(fb) * TC_PANEL_BYTES + 1024; }
static_assert(tc_smem_bytes(232) <= 227 * 1024 - 2048, "window stages fit the shared memory at the widest block");
static_assert(tc_tmem_cols(208, true) <= 512 && tc_tmem_cols(232, false) <= 512, "tensor-memory budget");

// All lanes wait on the barrier; the warp proceeds (converged) only if every
// lane saw the phase complete.
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity, volatile int *abort)
{
    const bool ok = mbar_wait(bar, parity, abort);
    return __all_sync(0xffffffffu, ok);
}

// One record of the stage ring.  kind: TC_STEP (chunk ch of an active
// step's window: step s, window start lo, nk 16-row chunks in the window),
// TC_END (end of item `it`, n records), TC_FINAL (no more items).  it counts
// the CTA's items.
enum TcKind : int32_t { TC_STEP = 0, TC_END = 1, TC_FINAL = 2 };
struct TcInfo {
    int32_t kind, s, lo, nk, ch, it, n, tx, rx;
};
// a record written by another thread (published through an mbarrier)
__device__ __forceinline__ TcInfo read_info(const TcInfo *p)
{
    const volatile TcInfo *v = p;
    TcInfo r;
    r.kind = v->kind; r.s = v->s; r.lo = v->lo; r.nk = v->nk; r.ch = v->ch; r.it = v->it; r.n = v->n;
    r.tx = v->tx; r.rx = v->rx;
    return r;
}

struct TcParams {
    CUtensorMap tmap;           // slab rows: dim 0 = 2 FB halfs (a row), dim 1 = rows of all slabs
    FusedJob job;
    int32_t fb;                 // frames per block (multiple of 8, 32..tc_max_fb)
    int32_t rows_per_slab;      // n_sample + 32 (zero rows past the record)
    int64_t s2_row0;            // first row of the (-im, re) slabs S' in the tensor map
    int64_t n_items;            // n_fb * tiles
    unsigned long long *err_count;
};

// Tile coordinates of a tile index, depth slowest: the CTAs working at one
// time hold tiles of one or two depths, whose windows of a step cover a few
// hundred of the slab's rows, so the rows they read stay in L2 while the
// CTAs drift apart across the steps.
__device__ __forceinline__ void tc_tile_coords(const FusedJob &J, int64_t tile, int &tu, int &tv, int &tz)
{
    tu = (int)(tile % J.tiles_u);
    tv = (int)((tile / J.tiles_u) % J.tiles_v);
    tz = (int)(tile / ((int64_t)J.tiles_u * J.tiles_v));
}

// One step's window for the tile (producer): rows [lo, lo + 16 nk) of the
// step's slab cover every tap of every voxel of the tile.
template <int KIND>
__device__ __forceinline__ bool tc_window(const FusedJob &J, int s, int tx, int rx, int tu, int tv, int tz, int &lo,
                                          int &nk, bool &overflow)
{
    using KT = KindTraits<KIND>;
    overflow = false;
    const float2 rr = J.rx_range[((int64_t)rx * J.tiles_u + tu) * J.tiles_z + tz];
    const float2 tr = J.tx_range[((int64_t)tx * J.tiles_v + tv) * J.tiles_z + tz];
    if (!(rr.x <= rr.y) || !(tr.x <= tr.y)) return false;
    const float ab = ab_value(J.g, tx, rx);
    float lo_f = __fadd_rn(__fadd_rn(tr.x, rr.x), ab);
    float hi_f = __fadd_rn(__fadd_rn(tr.y, rr.y), ab);
    const float fmax_n = (float)J.n_sample;
    lo_f = fminf(fmaxf(floorf(lo_f), -1.0f), fmax_n);
    hi_f = fminf(fmaxf(floorf(hi_f), -1.0f), fmax_n);
    int l = max((int)lo_f - KT::LO, 0);
    const int h = min((int)hi_f - KT::LO + KT::TAPS - 1, J.n_sample - 2);
    if (h < l) return false;
    const int count = h - l + 1;
    nk = (count + 15) >> 4;
    if (nk > TC_KCH) { overflow = true; return false; }
    lo = l;
    (void)s;
    return true;
}

// The TAPS weights shifted to start at position o of an NP-position row
// (positions outside the taps are zero): a barrel shifter of log2(NP)
// select stages, so that no register is indexed at run time.
template <int TAPS, int NP>
__device__ __forceinline__ void tc_place(const float (&w)[TAPS], int o, float (&v)[NP])
{
#pragma unroll
    for (int p = 0; p < NP; ++p) v[p] = p < TAPS ? w[p] : 0.0f;
#pragma unroll
    for (int b = 1; b < NP; b <<= 1) {
        const bool on = (o & b) != 0;
#pragma unroll
        for (int p = NP - 1; p >= 0; --p) v[p] = on ? (p >= b ? v[p - b] : 0.0f) : v[p];
    }
}

// FP32 values -> packed 16-bit pairs (even index in the low half), FP16 or
// (BF) BF16, the operand type of the slabs: the value's rounding (hi) and,
// for SPLIT, the rounding of the remainder (lo).
template <bool BF>
__device__ __forceinline__ uint32_t tc_pack(float a, float b)
{
    uint32_t r;
    if constexpr (BF) {
        __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        memcpy(&r, &h, 4);
    } else {
        __half2 h = __floats2half2_rn(a, b);
        memcpy(&r, &h, 4);
    }
    return r;
}
// x - hi for both halves as one packed FMA (hi * -1 + x: the subtraction's
// single rounding)
template <bool BF>
__device__ __forceinline__ uint32_t tc_pack_rem(float2 x, uint32_t hi)
{
    float2 f;
    if constexpr (BF) {
        __nv_bfloat162 h;
        memcpy(&h, &hi, 4);
        f = __bfloat1622float2(h);
    } else {
        __half2 h;
        memcpy(&h, &hi, 4);
        f = __half22float2(h);
    }
    const float2 r = __ffma2_rn(f, make_float2(-1.0f, -1.0f), x);
    return tc_pack<BF>(r.x, r.y);
}

// BF: BF16 slabs and weights (BF16 x BF16 MMAs; A and B of one MMA have the
// same type), else FP16
template <int KIND, bool SPLIT, bool BF>
__global__ void __launch_bounds__(TC_THREADS, 1) fused_tc_kernel(const __grid_constant__ TcParams prm)
{
    using KT = KindTraits<KIND>;
    constexpr int TAPS = KT::TAPS;
    constexpr int NMAT = tc_nmat(SPLIT);
    const FusedJob &J = prm.job;
    const DevGeom &g = J.g;
    const int FB = prm.fb;
    const int NH = 2 * FB;                 // halfs per slab row
    const int N16 = tc_n16(FB);            // accumulator columns
    const int NP = tc_panels(FB);
    const int chunk_bytes = NP * TC_PANEL_BYTES;   // 16 rows of S; the same rows of S' follow
    const int stage_bytes = 2 * chunk_bytes;
    const int a_col0 = N16;                // first weight-matrix column
    // one MMA per weight matrix covers columns [0, n_a); a second one
    // [TC_NMAX, N16) when the block is wider (its B operand starts at panel
    // TC_NMAX / 64)
    const int n_a = N16 < TC_NMAX ? N16 : TC_NMAX;
    const int n_b = N16 - n_a;
    const uint32_t idesc_a = idesc_f16_kmaj_a_mnmaj_b(128, n_a, BF);
    const uint32_t idesc_b = idesc_f16_kmaj_a_mnmaj_b(128, n_b > 0 ? n_b : 16, BF);

    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full_b[TC_NSB], empty_b[TC_NSB], full_a[TC_NSA], rec_full[TC_NSR], rec_empty[TC_NSR];
    __shared__ uint64_t acc_full, acc_empty, fin;
    __shared__ TcInfo info[TC_NSR];
    __shared__ volatile int last_rec[TC_NSB];   // loader: latest record loaded into each stage, -1 none
    __shared__ uint32_t tbase_s;
    __shared__ volatile int abort_s;
    __shared__ volatile int acc_seen;   // latest item whose accumulator phase a builder group has seen complete
    uint8_t *Bs = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        unsigned dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (dyn < (unsigned)tc_smem_bytes(FB) || tc_tmem_cols(FB, SPLIT) > 512 || NH < 64 || (FB & 7) ||
            J.compound == 0 || J.tu * J.tv != 128 || J.tz != 1) {
            if (tid == 0) atomicAdd(prm.err_count, 1ull);
            return;
        }
    }
    if (tid == 0) {
        for (int i = 0; i < TC_NSB; ++i) {
            mbar_init(&full_b[i], 1);
            mbar_init(&empty_b[i], 1);
        }
        for (int i = 0; i < TC_NSR; ++i) {
            mbar_init(&rec_full[i], 1);
            mbar_init(&rec_empty[i], 1);
        }
        for (int i = 0; i < TC_NSA; ++i) {
            mbar_init(&full_a[i], 128);
        }
        for (int i = 0; i < TC_NSB; ++i) last_rec[i] = -1;
        mbar_init(&acc_full, 1);
        mbar_init(&acc_empty, 128);
        mbar_init(&fin, 1);
        abort_s = 0;
        acc_seen = -1;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        tmem_alloc(&tbase_s, 512);
        tmem_relinquish();
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tb = tbase_s;
    volatile int *abort = &abort_s;

    const int64_t n_tiles = (int64_t)J.tiles_z * J.tiles_u * J.tiles_v;
    const int n_steps = g.n_tx * g.n_ele;

    if (warp == TC_PRODUCER_WARP) {
        // ---------------- producer: windows and records ----------------
        // The warp computes the windows of 32 steps at a time; each lane with
        // an active step then writes that step's chunk records itself (their
        // places in the ring follow the records of the lanes below), TC_NPUB
        // records at a time.  A record goes into its slot once the MMA warp
        // is done with the record TC_NSR earlier; the builders and the loader
        // pick it up from there.
        uint32_t q = 0;          // next record (warp-uniform)
        bool stop = false;       // warp-uniform after each batch
        auto emit = [&](uint32_t qr, const TcInfo rec) -> bool {
            const int rs = (int)(qr % TC_NSR);
            if (!mbar_wait(&rec_empty[rs], ((qr / TC_NSR) & 1u) ^ 1u, abort)) return false;
            info[rs] = rec;
            mbar_arrive(&rec_full[rs]);
            return true;
        };
        int it = 0;
        for (int64_t item = blockIdx.x; item < prm.n_items && !stop; item += gridDim.x, ++it) {
            const int64_t tile = item % n_tiles;
            int tu, tv, tz;
            tc_tile_coords(J, tile, tu, tv, tz);
            int n_active = 0;
            for (int s0 = 0; s0 < n_steps && !stop; s0 += 32) {
                const int s = s0 + lane;
                int lo = 0, nk = 0, tx = 0, rx = 0;
                bool act = false, ovf = false;
                if (s < n_steps) {
                    tx = s / g.n_ele;
                    rx = s - tx * g.n_ele;
                    act = tc_window<KIND>(J, s, tx, rx, tu, tv, tz, lo, nk, ovf);
                    if (ovf) atomicAdd(prm.err_count, 1ull);   // never expected: the planner bounds the window
                }
                // the step's chunk records follow the records of the lanes
                // below it (exclusive prefix sum of the chunk counts)
                const int cnt = act ? nk : 0;
                int incl = cnt;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, incl, d);
                    if (lane >= d) incl += v;
                }
                const int base = incl - cnt;
                const int n_rec = __shfl_sync(0xffffffffu, incl, 31);
                // in rounds of at most TC_NPUB records: a slot's barrier
                // tells apart only the phase of its previous use, so no lane
                // may wait on a slot more than one use ahead of the records
                // already written
                for (int r0 = 0; r0 < n_rec && !stop; r0 += TC_NPUB) {
                    bool ok = true;
                    for (int j = 0; j < cnt && ok; ++j) {
                        const int r = base + j;
                        if (r >= r0 && r < r0 + TC_NPUB)
                            ok = emit(q + (uint32_t)r, TcInfo{TC_STEP, s, lo, nk, j, it, 0, tx, rx});
                    }
                    stop = __any_sync(0xffffffffu, !ok);
                }
                q += (uint32_t)n_rec;
                n_active += n_rec;
            }
            if (!stop) {   // end of item
                bool ok = true;
                if (lane == 0) ok = emit(q, TcInfo{TC_END, 0, 0, 0, 0, it, n_active, 0, 0});
                stop = __any_sync(0xffffffffu, !ok);
                ++q;
            }
        }
        if (!stop) {   // one final record per builder group (TC_GROUPS <= TC_NPUB)
            bool ok = true;
            if (lane < TC_GROUPS) ok = emit(q + (uint32_t)lane, TcInfo{TC_FINAL, 0, 0, 0, 0, it, 0, 0, 0});
            stop = __any_sync(0xffffffffu, !ok);
        }
    } else if (warp == TC_LOADER_WARP) {
        // ---------------- loader: the records' rows, one record at a time ----------------
        // Record q's rows go into stage q mod TC_NSB once the MMAs of record
        // q - TC_NSB have completed; end records pass their stage on with no
        // copy.  The waits are in record order, so each stage's barrier is at
        // most one use behind the wait and its parity identifies the use.
        if (lane == 0) {
            tma_prefetch_desc(&prm.tmap);
            for (uint32_t q = 0;; ++q) {
                const int rs = (int)(q % TC_NSR), st = (int)(q % TC_NSB);
                if (!mbar_wait(&rec_full[rs], (q / TC_NSR) & 1u, abort)) break;
                const TcInfo inf = read_info(&info[rs]);
                if (inf.kind == TC_FINAL) break;
                if (!mbar_wait(&empty_b[st], ((q / TC_NSB) & 1u) ^ 1u, abort)) break;
                if (inf.kind == TC_STEP) {
                    const int64_t item = blockIdx.x + (int64_t)inf.it * gridDim.x;
                    const int64_t fb = item / n_tiles;
                    const int64_t row0 = ((int64_t)inf.s * J.n_fb + fb) * prm.rows_per_slab + inf.lo + 16 * inf.ch;
                    last_rec[st] = (int)q;
                    mbar_arrive_expect_tx(&full_b[st], (uint32_t)(2 * chunk_bytes));
                    uint8_t *dst = Bs + st * stage_bytes;
                    tma_load_3d(dst, &prm.tmap, &full_b[st], 0, (int32_t)row0, 0);
                    tma_load_3d(dst + chunk_bytes, &prm.tmap, &full_b[st], 0, (int32_t)(prm.s2_row0 + row0), 0);
                } else {
                    last_rec[st] = -1;   // no copy in flight
                    mbar_arrive(&full_b[st]);
                }
            }
            if (*abort) {
                // let the copies in flight land before the CTA's shared memory goes
                for (int st = 0; st < TC_NSB; ++st)
                    if (last_rec[st] >= 0) {
                        volatile int dummy = 0;
                        mbar_wait(&full_b[st], ((uint32_t)last_rec[st] / TC_NSB) & 1u, &dummy, 100000000ull);
                    }
            }
        }
    } else if (warp == TC_MMA_WARP) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            uint32_t q = 0;
            bool issued = false, first = true, dacc = false;
            for (;;) {
                const int bst = (int)(q % TC_NSB), rs = (int)(q % TC_NSR);
                if (!mbar_wait(&rec_full[rs], (q / TC_NSR) & 1u, abort)) break;
                const TcInfo inf = read_info(&info[rs]);
                if (inf.kind == TC_FINAL) break;
                if (!mbar_wait(&full_b[bst], (q / TC_NSB) & 1u, abort)) break;
                const int ast = (int)(q % TC_NSA);
                if (!mbar_wait(&full_a[ast], (q / TC_NSA) & 1u, abort)) break;
                ++q;
                // at an item's first record (its end record when no step is
                // active): the previous item's outputs have been read out, so
                // the accumulators may be overwritten or reported complete
                if (first) {
                    if (!mbar_wait(&acc_empty, ((uint32_t)inf.it & 1u) ^ 1u, abort)) break;
                    first = false;
                }
                if (inf.kind == TC_END) {
                    umma_commit(&acc_full);
                    // released once the MMAs issued so far have completed,
                    // like the stages of step records
                    umma_commit(&empty_b[bst]);
                    mbar_arrive(&rec_empty[rs]);
                    first = true;
                    dacc = false;
                    continue;
                }
                tmem_fence_after_sync();
                const uint32_t bbase = smem_u32(Bs + bst * stage_bytes);
                const uint32_t acol = (uint32_t)(a_col0 + ast * NMAT * 8);
                const uint32_t acc0 = dacc ? 1u : 0u;   // the item's first record starts the sums
#pragma unroll
                for (int mat = 0; mat < NMAT; ++mat) {
                    // Re(W) against S, Im(W) against S' = (-im, re)
                    const uint32_t b0 = bbase + (mat < NMAT / 2 ? 0u : (uint32_t)chunk_bytes);
                    const uint32_t acc = mat == 0 ? acc0 : 1u;
                    umma_f16_ts(tb, tb + acol + mat * 8, sdesc_mn_sw128(b0, TC_PANEL_BYTES, 1024), idesc_a, acc);
                    if (n_b > 0)
                        umma_f16_ts(tb + (uint32_t)TC_NMAX, tb + acol + mat * 8,
                                    sdesc_mn_sw128(b0 + (TC_NMAX / 64) * TC_PANEL_BYTES, TC_PANEL_BYTES, 1024),
                                    idesc_b, acc);
                }
                dacc = true;
                umma_commit(&empty_b[bst]);   // releases the stage and, for the builders, the weight slot
                mbar_arrive(&rec_empty[rs]);
                issued = true;
            }
            if (*abort && issued) {   // the MMAs in flight complete before the columns are freed
                umma_commit(&fin);
                volatile int dummy = 0;
                mbar_wait(&fin, 0, &dummy, 100000000ull);
            }
        }
    } else {
        // ---------------- weight builders + epilogue (warps 0 .. 4 TC_GROUPS - 1) ----------------
        const int grp = warp >> 2;
        const uint32_t lane_base = tb + ((uint32_t)(32 * (warp & 3)) << 16);
        const int m = tid & 127;            // voxel row of the tile = tensor-memory lane
        const int lu = m % J.tu, lv = m / J.tu;
        const int64_t n_rxkey = g.n_u * g.n_z, n_txkey = g.n_v * g.n_z;
        int cur_it = -1, fb = 0, cur_tx = -1, pre_s = -1;
        int64_t iz = 0, iu = 0, iv = 0, rxkey = 0, txkey = 0;
        bool valid = false, cone = false;
        float itx = 0.f, ptr = 0.f, pti = 0.f;
        float4 pre_e = make_float4(0.f, 0.f, 0.f, 0.f);
        for (uint32_t q = (uint32_t)grp;; q += TC_GROUPS) {
            const int rs = (int)(q % TC_NSR);
            if (!warp_wait(&rec_full[rs], (q / TC_NSR) & 1u, abort)) break;
            const TcInfo inf = read_info(&info[rs]);
            if (inf.kind == TC_FINAL) break;
            if (inf.it != cur_it) {   // a new item: this thread's voxel
                cur_it = inf.it;
                const int64_t item = blockIdx.x + (int64_t)inf.it * gridDim.x;
                fb = (int)(item / n_tiles);
                const int64_t tile = item % n_tiles;
                int tu, tv, tz;
                tc_tile_coords(J, tile, tu, tv, tz);
                iz = tz; iu = (int64_t)tu * J.tu + lu; iv = (int64_t)tv * J.tv + lv;
                valid = iz < g.n_z && iu < g.n_u && iv < g.n_v;
                rxkey = valid ? iu * g.n_z + iz : 0;
                txkey = valid ? iv * g.n_z + iz : 0;
                cur_tx = -1;
                pre_s = -1;
            }
            const int ast = (int)(q % TC_NSA);
            // the slot's previous use, record q - TC_NSA, has been consumed:
            // its MMAs completed, which the MMA warp signals (tcgen05.commit,
            // in record order) on the window stage that record used.  That
            // stage's barrier has completed the use before it, record
            // q - TC_NSA - TC_NSB (this group's previous record q - TC_GROUPS
            // waited for the later record q - TC_GROUPS - TC_NSA, as
            // TC_GROUPS <= TC_NSB), and not the use after it, record
            // q + TC_NSB - TC_NSA (its MMAs follow this record's), so the
            // parity identifies the use.
            auto wait_slot = [&]() -> bool {
                if (q < (uint32_t)TC_NSA) return true;
                const uint32_t qp = q - TC_NSA;
                return warp_wait(&empty_b[qp % TC_NSB], (qp / TC_NSB) & 1u, abort);
            };
            if (inf.kind == TC_END) {
                if (!wait_slot()) break;
                mbar_arrive(&full_a[ast]);
                // ---- epilogue: D -> out (frames of this block) ----
                // acc_full completes once per item.  Its parity names the
                // item only if the previous item's phase has completed: the
                // group of that item's end record has seen it.  (An item of
                // fewer than two records could otherwise reach this wait
                // while the phase of the item two back is still open.)
                bool seen = true;
                if (inf.it > 0 && acc_seen < inf.it - 1) {
                    const uint64_t t0 = global_ns();
                    while (acc_seen < inf.it - 1) {
                        if (*abort) { seen = false; break; }
                        if (global_ns() - t0 > 2000000000ull) { *abort = 1; seen = false; break; }
                    }
                }
                if (!__all_sync(0xffffffffu, seen)) break;
                if (!warp_wait(&acc_full, (uint32_t)inf.it & 1u, abort)) break;
                if (m == 0) acc_seen = inf.it;
                tmem_fence_after_sync();
                const int64_t pix = iz * g.s_z + iu * g.s_u + iv * g.s_v;
                for (int c = 0; c < N16; c += 16) {
                    uint32_t r[16];
                    tmem_ld16(lane_base + (uint32_t)c, r);
                    tmem_wait_ld16(r);
                    if (valid) {
#pragma unroll
                        for (int h = 0; h < 8; ++h) {
                            const int f = fb * FB + c / 2 + h;
                            if (c / 2 + h < FB && f < J.n_frame) {
                                float2 val = make_float2(0.f, 0.f);
                                if (inf.n > 0) {
                                    val.x = __uint_as_float(r[2 * h]) * (1.0f / TC_SCALE);
                                    val.y = __uint_as_float(r[2 * h + 1]) * (1.0f / TC_SCALE);
                                }
                                float2 *op = J.out + (int64_t)f * g.n_pix + pix;
                                if (J.accumulate) { float2 x = *op; x.x += val.x; x.y += val.y; *op = x; }
                                else *op = val;
                            }
                        }
                    }
                }
                tmem_fence_before_sync();
                mbar_arrive(&acc_empty);
                continue;
            }
            const int tx = inf.tx, rx = inf.rx;
            if (tx != cur_tx) {
                cur_tx = tx;
                const float4 t = valid ? __ldg(&g.tx_tab[(int64_t)tx * n_txkey + txkey])
                                       : make_float4(0.f, 0.f, 0.f, 0.f);
                itx = t.x; ptr = t.y; pti = t.z;
                cone = valid && t.w != 0.0f && (g.cone_u == nullptr || g.cone_u[(int64_t)tx * n_rxkey + rxkey] != 0);
            }
            float4 e;
            if (pre_s == inf.s) e = pre_e;
            else e = valid ? __ldg(&g.rx_tab[(int64_t)rx * n_rxkey + rxkey]) : make_float4(0.f, 0.f, 0.f, 0.f);
            // the receive entry of this group's next record is loaded while
            // this one is built: that record's step when the producer has
            // written it already (a test, no wait), else a guess three
            // steps on
            {
                const uint32_t qn = q + TC_GROUPS;
                const int rn = (int)(qn % TC_NSR);
                int ns = inf.s + TC_GROUPS, nrx = rx + TC_GROUPS;
                if (mbar_test_wait(&rec_full[rn], (qn / TC_NSR) & 1u)) {
                    const volatile TcInfo *v = &info[rn];
                    if (v->kind == TC_STEP) { ns = v->s; nrx = v->rx; }
                }
                if (valid && nrx < g.n_ele) {
                    pre_s = ns;
                    pre_e = __ldg(&g.rx_tab[(int64_t)nrx * n_rxkey + rxkey]);
                } else {
                    pre_s = -1;
                }
            }
            const float ab = ab_value(g, tx, rx);
            const float2 abp = ab_phasor(g, tx, rx);
            const float idx = __fadd_rn(__fadd_rn(itx, e.x), ab);
            const float fl = floorf(idx);
            bool ok = cone && e.w > 0.0f && fl >= (float)KT::LO && fl < (float)(J.n_sample - 1 - KT::HI);
            int o = ok ? (int)fl - KT::LO - inf.lo : 0;
            if (ok && (o < 0 || o + TAPS > 16 * inf.nk)) {   // never expected: window bound violated
                atomicAdd(prm.err_count, 1ull);
                ok = false;
                o = 0;
            }
            // a warp none of whose voxels has a tap in this record stores
            // zero rows without forming weights
            const bool warp_any = __any_sync(0xffffffffu, ok);
            float w[TAPS];
            if (warp_any) poly_weights<KIND, 6>(ok ? idx - fl : 0.0f, w);
            // P = apod e^{j phi_tx} e^{j phi_rx} e^{j phi_ab} (apod folded in (ar, ai)), scaled
            const float qx = fmaf(ptr, e.y, -pti * e.z), qy = fmaf(ptr, e.z, pti * e.y);
            const float px = ok ? TC_SCALE * fmaf(qx, abp.x, -qy * abp.y) : 0.0f;
            const float py = ok ? TC_SCALE * fmaf(qx, abp.y, qy * abp.x) : 0.0f;
            const uint32_t acol = lane_base + (uint32_t)(a_col0 + ast * NMAT * 8);
            // the packed weight rows are formed in registers first; the wait
            // for the slot comes only before the stores, so that a group's
            // arithmetic overlaps the MMAs still reading the slot
            auto build = [&](auto wide) -> bool {
                constexpr bool WIDE = decltype(wide)::value;
                // the voxel's taps in this record's 16 rows: at o in a
                // one-chunk window; in a two-chunk window at o - 16 ch,
                // clipped to the chunk (placed at o + 16 - 16 ch over 32
                // positions, of which the upper 16 are kept; a start past
                // the end leaves the chunk empty)
                uint32_t words[NMAT][8];
#pragma unroll
                for (int mat = 0; mat < NMAT; ++mat)
#pragma unroll
                    for (int c = 0; c < 8; ++c) words[mat][c] = 0u;
                if (warp_any) {
                    float v[16];
                    if constexpr (WIDE) {
                        const int e = o + 16 - 16 * inf.ch;
                        float v32[32];
                        tc_place<TAPS, 32>(w, e < 32 ? e : 0, v32);
#pragma unroll
                        for (int p = 0; p < 16; ++p) v[p] = v32[16 + p];
                    } else {
                        tc_place<TAPS, 16>(w, o, v);
                    }
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        // (Re, Im) of the pair's two weights: packed FP32 products
                        const float2 vv = make_float2(v[2 * c], v[2 * c + 1]);
                        const float2 r = __fmul2_rn(vv, make_float2(px, px));
                        const float2 i = __fmul2_rn(vv, make_float2(py, py));
                        if constexpr (SPLIT) {
                            words[0][c] = tc_pack<BF>(r.x, r.y);
                            words[1][c] = tc_pack_rem<BF>(r, words[0][c]);
                            words[2][c] = tc_pack<BF>(i.x, i.y);
                            words[3][c] = tc_pack_rem<BF>(i, words[2][c]);
                        } else {
                            words[0][c] = tc_pack<BF>(r.x, r.y);
                            words[1][c] = tc_pack<BF>(i.x, i.y);
                        }
                    }
                }
                if (!wait_slot()) return false;
                tmem_fence_after_sync();
#pragma unroll
                for (int mat = 0; mat < NMAT; ++mat) tmem_st8(acol + (uint32_t)(mat * 8), words[mat]);
                tmem_wait_st();
                tmem_fence_before_sync();
                return true;
            };
            const bool built = inf.nk == 1 ? build(std::false_type{}) : build(std::true_type{});
            if (!built) break;
            mbar_arrive(&full_a[ast]);
        }
    }
    if (tid == 0 && *abort) atomicAdd(prm.err_count, 1ull);
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after_sync();
        tmem_dealloc(tb, 512);
    }
}

}  // namespace rcabf
