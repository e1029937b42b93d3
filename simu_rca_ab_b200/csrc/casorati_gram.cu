// Casorati Gram matrix of the SVD clutter filter on the tensor cores
// (tcgen05.mma kind::i8): the G = C^H C step of SVDClutterFilter.m:23-25
// (MATLAB/lib/clutterFilter/SVDClutterFilter.m), which the reference forms in
// double precision.
//
// x holds nT frames of n_pix complex pixels ([frame][pixel], pixel fastest:
// the beamformer's ensemble layout, the transpose of MATLAB's Casorati
// matrix C = reshape(IQ, [], nT)).  With y the 2 nT x n_pix real matrix whose
// row 2t is Re x_t and row 2t+1 is Im x_t, the real symmetric Y = y y^T gives
//     Re G[i][j] = Y[2i][2j] + Y[2i+1][2j+1]
//     Im G[i][j] = Y[2i][2j+1] - Y[2i+1][2j]
// with G[i][j] = sum_p conj(x[i][p]) x[j][p] = (C' * C)(i, j).
//
// Precision: an Ozaki-type split into integer slices.  The pixels are cut
// into chunks of cv voxels.  Per (row, chunk) every value is scaled by the
// power of two 2^(6-e) that brings the chunk's largest magnitude below 64,
// and the scaled value r is written as four signed 7-bit slices:
//     d0 = rint(r), d1 = rint(128 (r - d0)), ... (|d_s| <= 64), so that
//     y = 2^(e-6) (d0 + 2^-7 d1 + 2^-14 d2 + 2^-21 d3) + rest,
//     |rest| <= 2^(e-28) (at most 2^-27 of the chunk's largest magnitude).
// The tensor cores form the slice products exactly (int8 x int8 -> int32):
// per chunk and level n = s + t,
//     A_n = sum_{s + t = n} D_s D_t^T     (|A_n| <= 4 * 64^2 * cv < 2^31),
// and the chunk's share of Y is 2^(e_r + e_c - 12) sum_{n <= 4} 2^-7n A_n,
// formed in FP64.  Levels 5 and 6 (slice pairs (2,3), (3,2), (3,3)) are
// dropped; they sit 2^-35 below the leading term.  Chunks are summed in FP64
// in chunk order, so the result does not depend on scheduling.
//
// Kernels:
//   gram_slice_kernel   one CTA per (chunk, frame): the chunk's largest
//                       |Re| and |Im|, then the four slices of both rows
//                       (HBM-bound: reads x twice, the second time from L2,
//                       writes 4 bytes per value)
//   gram_mma_kernel     one CTA per (chunk, tile of Y): 128 rows (M) x nb
//                       columns (N) of Y, five int32 accumulators in tensor
//                       memory (one per level), 4-stage TMA pipeline of
//                       64-voxel K steps (all four slices of both row blocks
//                       per stage, 64-byte swizzle), 26 MMAs of K = 32 per
//                       stage; epilogue combines the levels in FP64 into the
//                       chunk's partial tile
//   gram_reduce_kernel  sums the partial tiles over the chunks into Y
//   gram_assemble_kernel  G (complex128, nT x nT) from Y's upper triangle
// Only tiles that meet Y's upper triangle are formed (Y is symmetric).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "../../include/rcabf.h"
#include "launchers.h"
#include "tc_common.cuh"

namespace rcabf {
namespace {

constexpr int GS_THREADS = 512;            // slicing CTA
constexpr int GM_THREADS = 128;            // MMA CTA: warp 0 lane 0 TMA, warp 1 lane 0 MMA, all four the epilogue
constexpr int GM_STAGES = 4;
constexpr int GM_KV = 64;                  // voxels (bytes of a slice row) per K step
constexpr int GM_M = 128;                  // rows of Y per tile (MMA M)
constexpr int GM_NMAX = 96;                // largest column block (MMA N)
constexpr int GM_SLICES = 4;
constexpr int GM_LEVELS = 5;               // levels 0..4 of slice pairs
constexpr int GM_COLSTRIDE = 96;           // tensor-memory columns between level accumulators
constexpr int GM_A_BYTES = GM_SLICES * GM_M * GM_KV;        // 32 KB
constexpr int GM_B_BYTES = GM_SLICES * GM_NMAX * GM_KV;     // 24 KB (largest)
constexpr int GM_STAGE_BYTES = GM_A_BYTES + GM_B_BYTES;
constexpr size_t GM_SMEM = (size_t)GM_STAGES * GM_STAGE_BYTES + 1024;
constexpr int GM_MAX_CV = 65536;           // keeps every level sum inside int32
constexpr int GM_DEFAULT_CV = 16384;
static_assert(GM_LEVELS * GM_COLSTRIDE <= 512, "level accumulators exceed tensor memory");
static_assert(GM_SMEM <= 232448, "pipeline exceeds shared memory");

struct GramParams {
    CUtensorMap qa;          // slices as [slice][row][voxel] bytes; box 64 voxels x 128 rows x 4 slices
    CUtensorMap qb;          // same tensor; box 64 voxels x nb rows x 4 slices
    const int32_t *ex;       // [rows][n_chunks] scale exponents
    double *part;            // [n_chunks][n_tiles][nb][128] partial tiles (column-major)
    unsigned long long *err;
    int64_t n_pix;
    int32_t rows;            // 2 nT
    int32_t n_chunks, cv, nb, n_i, n_j, n_tiles;
};

// Tile `idx` of the upper-triangle walk: column block J ascending, within it
// row blocks I = 0 .. min(n_i - 1, last row block meeting columns <= the
// block's last column).
__host__ __device__ inline void gram_tile_of(int idx, int nb, int n_i, int n_j, int &I, int &J)
{
    for (int j = 0; j < n_j; ++j) {
        const int last = (nb * j + nb - 1) / GM_M;
        const int cnt = (last < n_i - 1 ? last : n_i - 1) + 1;
        if (idx < cnt) {
            I = idx;
            J = j;
            return;
        }
        idx -= cnt;
    }
    I = J = 0;
}

__host__ __device__ inline int gram_tile_count(int nb, int n_i, int n_j)
{
    int n = 0;
    for (int j = 0; j < n_j; ++j) {
        const int last = (nb * j + nb - 1) / GM_M;
        n += (last < n_i - 1 ? last : n_i - 1) + 1;
    }
    return n;
}

// -------------------------------------------------------------------------
// slicing
// -------------------------------------------------------------------------
// exponent e with m < 2^e (m >= 2^(e-1)), or the flag that the chunk row is
// treated as zero (largest magnitude below 2^-100, or zero)
__device__ __forceinline__ int gram_exponent(float m, bool &zero)
{
    const uint32_t E = (__float_as_uint(m) >> 23) & 0xffu;
    int e = (int)E - 126;
    zero = (E == 0u) || e < -100;
    if (E == 0xffu) e = 129;   // Inf / NaN input: slices saturate, the Gram is meaningless
    return zero ? 0 : e;
}

// four 7-bit slices of r (|r| < 64 after scaling) into byte k of w[0..3]
__device__ __forceinline__ void gram_slices(float r, uint32_t (&w)[GM_SLICES], int k)
{
#pragma unroll
    for (int s = 0; s < GM_SLICES; ++s) {
        const float d = rintf(r);
        w[s] |= ((uint32_t)__float2int_rz(d) & 0xffu) << (8 * k);
        r = (r - d) * 128.0f;
    }
}

__global__ void __launch_bounds__(GS_THREADS) gram_slice_kernel(int8_t *__restrict__ Q, int32_t *__restrict__ ex,
                                                               const float2 *__restrict__ x, int64_t ld,
                                                               int64_t n_pix, int64_t vp, int rows, int cv,
                                                               int n_chunks)
{
    const int c = blockIdx.x, t = blockIdx.y;
    const int64_t v0 = (int64_t)c * cv, v1 = min(n_pix, v0 + cv);
    const float2 *row = x + (int64_t)t * ld;
    float mr = 0.f, mi = 0.f;
    for (int64_t v = v0 + threadIdx.x; v < v1; v += GS_THREADS) {
        const float2 a = row[v];
        mr = fmaxf(mr, fabsf(a.x));
        mi = fmaxf(mi, fabsf(a.y));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        mr = fmaxf(mr, __shfl_xor_sync(0xffffffffu, mr, o));
        mi = fmaxf(mi, __shfl_xor_sync(0xffffffffu, mi, o));
    }
    __shared__ float red[2][GS_THREADS / 32];
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = mr;
        red[1][threadIdx.x >> 5] = mi;
    }
    __syncthreads();
    mr = 0.f;
    mi = 0.f;
#pragma unroll
    for (int w = 0; w < GS_THREADS / 32; ++w) {
        mr = fmaxf(mr, red[0][w]);
        mi = fmaxf(mi, red[1][w]);
    }
    bool zr, zi;
    const int er = gram_exponent(mr, zr), ei = gram_exponent(mi, zi);
    // 2^(6 - e): biased exponent 133 - e in [4, 233], a normal float
    const float sr = zr ? 0.f : __uint_as_float((uint32_t)(133 - er) << 23);
    const float si = zi ? 0.f : __uint_as_float((uint32_t)(133 - ei) << 23);
    int8_t *qr = Q + (int64_t)(2 * t) * vp, *qi = Q + (int64_t)(2 * t + 1) * vp;
    const int64_t slice_stride = (int64_t)rows * vp;
    for (int64_t v = v0 + 4 * (int64_t)threadIdx.x; v < v1; v += 4 * GS_THREADS) {
        uint32_t wr[GM_SLICES] = {0u, 0u, 0u, 0u}, wi[GM_SLICES] = {0u, 0u, 0u, 0u};
        const int n = v1 - v < 4 ? (int)(v1 - v) : 4;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (k < n) {
                const float2 a = row[v + k];
                gram_slices(a.x * sr, wr, k);
                gram_slices(a.y * si, wi, k);
            }
        if (n == 4) {   // v is a multiple of 4 and vp of 16: aligned words
#pragma unroll
            for (int s = 0; s < GM_SLICES; ++s) {
                *reinterpret_cast<uint32_t *>(qr + s * slice_stride + v) = wr[s];
                *reinterpret_cast<uint32_t *>(qi + s * slice_stride + v) = wi[s];
            }
        } else {
            for (int k = 0; k < n; ++k)
#pragma unroll
                for (int s = 0; s < GM_SLICES; ++s) {
                    qr[s * slice_stride + v + k] = (int8_t)(wr[s] >> (8 * k));
                    qi[s * slice_stride + v + k] = (int8_t)(wi[s] >> (8 * k));
                }
        }
    }
    if (threadIdx.x == 0) {
        ex[(int64_t)(2 * t) * n_chunks + c] = er;
        ex[(int64_t)(2 * t + 1) * n_chunks + c] = ei;
    }
}

// -------------------------------------------------------------------------
// tensor-core Gram of one (chunk, tile)
// -------------------------------------------------------------------------
// K-major operand, 64-byte swizzle (atoms of 8 rows x 64 bytes, 512 bytes,
// 512-byte aligned): stride offset = 512 bytes between 8-row groups; the
// leading offset is unused (one MMA's K of 32 bytes lies inside a row).
__device__ __forceinline__ uint64_t sdesc_kmaj_sw64(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | ((uint64_t)(512 >> 4) << 32) | (1ull << 46) |
           (4ull << 61);
}
// kind::i8, signed x signed -> int32, both operands K-major, M x N
__device__ __forceinline__ uint32_t idesc_i8(int m, int n)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
// D[tmem] (+)= A[smem desc] * B[smem desc]^T, kind::i8, single CTA
__device__ __forceinline__ void umma_i8_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                           uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ double pow2d(int k)   // 2^k, k in the normal range
{
    return __longlong_as_double((long long)(1023 + k) << 52);
}

__global__ void __launch_bounds__(GM_THREADS, 1) gram_mma_kernel(const __grid_constant__ GramParams p)
{
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full[GM_STAGES], empty[GM_STAGES], acc_full;
    __shared__ uint32_t tbase_s;
    __shared__ volatile int abort_s;
    __shared__ int issued_s, consumed_s;   // K steps loaded / consumed by the MMAs
    uint8_t *sm = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        unsigned dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (dyn < (unsigned)GM_SMEM || p.nb > GM_NMAX || (p.nb & 15) || p.nb < 16) {
            if (tid == 0) atomicAdd(p.err, 1ull);
            return;
        }
    }
    const int tile = (int)(blockIdx.x % (unsigned)p.n_tiles), chunk = (int)(blockIdx.x / (unsigned)p.n_tiles);
    int I, J;
    gram_tile_of(tile, p.nb, p.n_i, p.n_j, I, J);
    const int n_eff = min(p.nb, (p.rows - p.nb * J + 15) & ~15);   // MMA N: the block's rows, rounded to 16
    const int64_t v0 = (int64_t)chunk * p.cv;
    const int64_t kv = p.n_pix - v0 < p.cv ? p.n_pix - v0 : (int64_t)p.cv;
    const int nk = (int)((kv + GM_KV - 1) / GM_KV);
    const uint32_t b_slice = (uint32_t)p.nb * GM_KV;   // bytes between slices in the B tile (512-byte multiple)

    if (tid == 0) {
        for (int i = 0; i < GM_STAGES; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(&acc_full, 1);
        abort_s = 0;
        issued_s = consumed_s = 0;
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

    if (warp == 0 && lane == 0) {
        // ---------------- producer ----------------
        tma_prefetch_desc(&p.qa);
        tma_prefetch_desc(&p.qb);
        const uint32_t bytes = (uint32_t)GM_A_BYTES + GM_SLICES * b_slice;
        int k = 0;
        for (; k < nk; ++k) {
            const int st = k % GM_STAGES, u = k / GM_STAGES;
            if (u > 0 && !mbar_wait(&empty[st], (uint32_t)(u - 1) & 1u, abort)) break;
            uint8_t *a = sm + (size_t)st * GM_STAGE_BYTES;
            mbar_arrive_expect_tx(&full[st], bytes);
            const int32_t xv = (int32_t)(v0 + (int64_t)k * GM_KV);   // multiple of 64 bytes
            tma_load_3d(a, &p.qa, &full[st], xv, GM_M * I, 0);
            tma_load_3d(a + GM_A_BYTES, &p.qb, &full[st], xv, p.nb * J, 0);
        }
        issued_s = k;
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer ----------------
        const uint32_t idesc = idesc_i8(GM_M, n_eff);
        int k = 0;
        for (; k < nk; ++k) {
            const int st = k % GM_STAGES, u = k / GM_STAGES;
            if (!mbar_wait(&full[st], (uint32_t)u & 1u, abort)) break;
            tmem_fence_after_sync();
            const uint32_t a0 = smem_u32(sm + (size_t)st * GM_STAGE_BYTES), b0 = a0 + GM_A_BYTES;
#pragma unroll
            for (int n = 0; n < GM_LEVELS; ++n) {
                const int s_lo = n > GM_SLICES - 1 ? n - (GM_SLICES - 1) : 0;
                const int s_hi = n < GM_SLICES - 1 ? n : GM_SLICES - 1;
#pragma unroll
                for (int s = s_lo; s <= s_hi; ++s)
#pragma unroll
                    for (int kk = 0; kk < GM_KV / 32; ++kk) {
                        const uint64_t ad = sdesc_kmaj_sw64(a0 + (uint32_t)s * (GM_M * GM_KV) + 32u * kk);
                        const uint64_t bd = sdesc_kmaj_sw64(b0 + (uint32_t)(n - s) * b_slice + 32u * kk);
                        umma_i8_ss(tb + (uint32_t)(n * GM_COLSTRIDE), ad, bd, idesc,
                                   (k > 0 || s > s_lo || kk > 0) ? 1u : 0u);
                    }
            }
            umma_commit(&empty[st]);
        }
        consumed_s = k;
        umma_commit(&acc_full);   // every MMA issued above, also after an abort
    }
    __syncwarp();

    // ---------------- epilogue: levels -> FP64 partial tile ----------------
    bool ok = mbar_wait(&acc_full, 0u, abort);
    ok = __all_sync(0xffffffffu, ok) && !*abort && nk > 0;
    if (ok) {
        tmem_fence_after_sync();
        const int i = 32 * warp + lane;                  // row of the tile (tensor-memory lane)
        const int r = GM_M * I + i;
        const int er = r < p.rows ? p.ex[(int64_t)r * p.n_chunks + chunk] : 0;
        double *out = p.part + ((int64_t)chunk * p.n_tiles + tile) * (int64_t)p.nb * GM_M;
        const uint32_t lane_base = tb + ((uint32_t)(32 * warp) << 16);
        for (int g = 0; g < n_eff / 16; ++g) {
            uint32_t v[GM_LEVELS][16];
#pragma unroll
            for (int n = 0; n < GM_LEVELS; ++n) tmem_ld16(lane_base + (uint32_t)(n * GM_COLSTRIDE + 16 * g), v[n]);
#pragma unroll
            for (int n = 0; n < GM_LEVELS; ++n) tmem_wait_ld16(v[n]);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int c = p.nb * J + 16 * g + j;
                const int ec = c < p.rows ? __ldg(p.ex + (int64_t)c * p.n_chunks + chunk) : 0;
                double s = (double)(int32_t)v[0][j];
#pragma unroll
                for (int n = 1; n < GM_LEVELS; ++n) s += (double)(int32_t)v[n][j] * pow2d(-7 * n);
                out[(int64_t)(16 * g + j) * GM_M + i] = s * pow2d(er + ec - 12);
            }
        }
    }
    if (tid == 0 && (*abort || !ok) && nk > 0) atomicAdd(p.err, 1ull);
    tmem_fence_before_sync();
    __syncthreads();
    if (tid == 0) {
        // after an abort: loads still in flight land before the CTA's shared
        // memory is released (bounded waits)
        volatile int stop = 0;
        for (int k = consumed_s; k < issued_s; ++k)
            if (!mbar_wait(&full[k % GM_STAGES], (uint32_t)(k / GM_STAGES) & 1u, &stop)) break;
    }
    if (warp == 0) {
        tmem_fence_after_sync();
        tmem_dealloc(tb, 512);
    }
}

// Y[a][b] = sum over chunks (in order) of the partial tiles, for every (a, b)
// of a formed tile inside the 2 nT x 2 nT matrix
__global__ void gram_reduce_kernel(double *__restrict__ Y, const double *__restrict__ part, int rows, int n_chunks,
                                   int nb, int n_i, int n_j, int n_tiles)
{
    const int64_t per_tile = (int64_t)nb * GM_M;
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= per_tile * n_tiles) return;
    const int tile = (int)(idx / per_tile);
    const int j = (int)((idx % per_tile) / GM_M), i = (int)(idx % GM_M);
    int I, J;
    gram_tile_of(tile, nb, n_i, n_j, I, J);
    const int a = GM_M * I + i, b = nb * J + j;
    if (a >= rows || b >= rows) return;
    double s = 0.0;
    for (int c = 0; c < n_chunks; ++c) s += part[((int64_t)c * n_tiles + tile) * per_tile + (int64_t)j * GM_M + i];
    Y[(int64_t)a * rows + b] = s;
}

__device__ __forceinline__ double gram_y(const double *Y, int rows, int a, int b)
{
    return a <= b ? Y[(int64_t)a * rows + b] : Y[(int64_t)b * rows + a];
}

// G[i][j] (complex128, row-major) from the upper triangle of Y
__global__ void gram_assemble_kernel(double2 *__restrict__ G, const double *__restrict__ Y, int nt)
{
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)nt * nt) return;
    const int i = (int)(idx / nt), j = (int)(idx % nt), rows = 2 * nt;
    const double re = gram_y(Y, rows, 2 * i, 2 * j) + gram_y(Y, rows, 2 * i + 1, 2 * j + 1);
    const double im = gram_y(Y, rows, 2 * i, 2 * j + 1) - gram_y(Y, rows, 2 * i + 1, 2 * j);
    G[idx] = make_double2(re, im);
}

static PFN_cuTensorMapEncodeTiled_v12000 gram_tensor_map_encoder()
{
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void *q = nullptr;
        cudaDriverEntryPointQueryResult r;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &q, cudaEnableDefault, &r) == cudaSuccess &&
            r == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(q);
    });
    return fn;
}

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

struct GramPlan {
    int64_t nt = 0, n_pix = 0, vp = 0;
    int rows = 0, cv = 0, n_chunks = 0, nb = 0, n_i = 0, n_j = 0, n_tiles = 0;
    size_t off_q = 0, off_e = 0, off_part = 0, off_y = 0, bytes = 0;
    double int_ops = 0.0;   // 2 x multiply-adds the tensor cores perform
};

// Column block nb in {64, 80, 96}: the fewest tile-stages, each priced at the
// larger of its MMA time (13 N cycles) and its load time (bytes / 40 B per
// cycle, an estimate of one SM's share of L2 bandwidth).
static int gram_plan(int64_t nt, int64_t n_pix, int32_t chunk_voxels, GramPlan &g)
{
    if (nt < 1 || n_pix < 1) return RCABF_ERR_SHAPE_MISMATCH;
    if (nt > 16384) return RCABF_ERR_UNSUPPORTED;
    int cv = chunk_voxels > 0 ? chunk_voxels : GM_DEFAULT_CV;
    if (cv % GM_KV || cv > GM_MAX_CV) return RCABF_ERR_INVALID_ARGUMENT;
    g.nt = nt;
    g.n_pix = n_pix;
    g.rows = (int)(2 * nt);
    g.vp = (n_pix + 15) & ~(int64_t)15;
    g.cv = cv;
    const int64_t n_chunks = (n_pix + cv - 1) / cv;
    if (n_chunks > INT32_MAX / 4 || n_pix > ((int64_t)1 << 31) - GM_MAX_CV) return RCABF_ERR_UNSUPPORTED;
    g.n_chunks = (int)n_chunks;
    g.n_i = (g.rows + GM_M - 1) / GM_M;
    double best = 0.0;
    for (int nb : {64, 80, 96}) {
        const int n_j = (g.rows + nb - 1) / nb;
        const int tiles = gram_tile_count(nb, g.n_i, n_j);
        const double cost = tiles * std::max(13.0 * nb, (GM_M + nb) * 4.0 * GM_KV / 40.0);
        if (g.nb == 0 || cost < best) {
            best = cost;
            g.nb = nb;
            g.n_j = n_j;
            g.n_tiles = tiles;
        }
    }
    if ((int64_t)g.n_tiles * g.n_chunks > INT32_MAX) return RCABF_ERR_UNSUPPORTED;
    g.off_q = 0;
    g.off_e = align256(g.off_q + (size_t)GM_SLICES * g.rows * g.vp);
    g.off_part = align256(g.off_e + (size_t)g.rows * g.n_chunks * sizeof(int32_t));
    g.off_y = align256(g.off_part + (size_t)g.n_chunks * g.n_tiles * g.nb * GM_M * sizeof(double));
    g.bytes = align256(g.off_y + (size_t)g.rows * g.rows * sizeof(double));
    // 13 slice pairs x 128 x N_eff x the K steps of every chunk
    double mac = 0.0;
    for (int t = 0; t < g.n_tiles; ++t) {
        int I, J;
        gram_tile_of(t, g.nb, g.n_i, g.n_j, I, J);
        const int n_eff = std::min(g.nb, (g.rows - g.nb * J + 15) & ~15);
        mac += 13.0 * GM_M * n_eff;
    }
    int64_t ksteps = 0;
    for (int64_t c = 0; c < g.n_chunks; ++c) ksteps += (std::min<int64_t>(n_pix - c * cv, cv) + GM_KV - 1) / GM_KV;
    g.int_ops = 2.0 * mac * (double)ksteps * GM_KV;
    return RCABF_OK;
}

}  // namespace
}  // namespace rcabf

using namespace rcabf;

extern "C" int rcabf_casorati_gram_plan(int64_t n_frame, int64_t n_pix, int32_t chunk_voxels,
                                        rcabf_gram_plan *out)
{
    if (!out || out->struct_size < (int32_t)sizeof(rcabf_gram_plan)) return RCABF_ERR_INVALID_ARGUMENT;
    GramPlan g;
    const int s = gram_plan(n_frame, n_pix, chunk_voxels, g);
    if (s != RCABF_OK) return s;
    out->workspace_bytes = g.bytes;
    out->chunk_voxels = g.cv;
    out->n_chunks = g.n_chunks;
    out->column_block = g.nb;
    out->n_tiles = g.n_tiles;
    out->mma_int_ops = g.int_ops;
    out->launches = 4;
    return RCABF_OK;
}

extern "C" int rcabf_casorati_gram(void *G, const void *x, int64_t n_frame, int64_t n_pix, int64_t ld,
                                   int32_t chunk_voxels, void *workspace, size_t workspace_bytes, void *stream)
{
    if (!G || !x || !workspace) return RCABF_ERR_INVALID_ARGUMENT;
    if (ld < n_pix) return RCABF_ERR_SHAPE_MISMATCH;
    if (((uintptr_t)x & 7u) || ((uintptr_t)G & 15u) || ((uintptr_t)workspace & 255u))
        return RCABF_ERR_INVALID_ARGUMENT;
    GramPlan g;
    int s = gram_plan(n_frame, n_pix, chunk_voxels, g);
    if (s != RCABF_OK) return s;
    if (workspace_bytes < g.bytes) return RCABF_ERR_INVALID_ARGUMENT;
    auto enc = gram_tensor_map_encoder();
    if (!enc) return RCABF_ERR_UNSUPPORTED;
    unsigned long long *err = current_error_counter();
    if (!err) return RCABF_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    uint8_t *ws = static_cast<uint8_t *>(workspace);
    int8_t *Q = reinterpret_cast<int8_t *>(ws + g.off_q);
    int32_t *ex = reinterpret_cast<int32_t *>(ws + g.off_e);
    double *part = reinterpret_cast<double *>(ws + g.off_part);
    double *Y = reinterpret_cast<double *>(ws + g.off_y);

    GramParams p{};
    // slices as a 3-D byte tensor: x = voxel (extent n_pix: voxels past it
    // read as zeros), y = row (extent 2 nT: rows past it read as zeros),
    // z = slice
    cuuint64_t dims[3] = {(cuuint64_t)g.n_pix, (cuuint64_t)g.rows, (cuuint64_t)GM_SLICES};
    cuuint64_t strides[2] = {(cuuint64_t)g.vp, (cuuint64_t)g.vp * g.rows};
    cuuint32_t box_a[3] = {GM_KV, GM_M, GM_SLICES}, box_b[3] = {GM_KV, (cuuint32_t)g.nb, GM_SLICES};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult cr = enc(&p.qa, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, Q, dims, strides, box_a, es,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr == CUDA_SUCCESS)
        cr = enc(&p.qb, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, Q, dims, strides, box_b, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                 CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return RCABF_ERR_INVALID_ARGUMENT;
    p.ex = ex;
    p.part = part;
    p.err = err;
    p.n_pix = g.n_pix;
    p.rows = g.rows;
    p.n_chunks = g.n_chunks;
    p.cv = g.cv;
    p.nb = g.nb;
    p.n_i = g.n_i;
    p.n_j = g.n_j;
    p.n_tiles = g.n_tiles;

    cudaError_t e = cudaFuncSetAttribute(gram_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)GM_SMEM);
    if (e != cudaSuccess) return RCABF_ERR_CUDA;
    gram_slice_kernel<<<dim3((unsigned)g.n_chunks, (unsigned)n_frame), GS_THREADS, 0, st>>>(
        Q, ex, static_cast<const float2 *>(x), ld, g.n_pix, g.vp, g.rows, g.cv, g.n_chunks);
    gram_mma_kernel<<<(unsigned)(g.n_tiles * g.n_chunks), GM_THREADS, GM_SMEM, st>>>(p);
    const int64_t nred = (int64_t)g.n_tiles * g.nb * GM_M;
    gram_reduce_kernel<<<(unsigned)((nred + 255) / 256), 256, 0, st>>>(Y, part, g.rows, g.n_chunks, g.nb, g.n_i,
                                                                     g.n_j, g.n_tiles);
    const int64_t ng = n_frame * n_frame;
    gram_assemble_kernel<<<(unsigned)((ng + 255) / 256), 256, 0, st>>>(static_cast<double2 *>(G), Y, (int)n_frame);
    count_launches(4);
    e = cudaGetLastError();
    return e == cudaSuccess ? RCABF_OK : RCABF_ERR_CUDA;
}
