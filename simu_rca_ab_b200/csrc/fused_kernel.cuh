// Fused persistent delay-and-sum kernel (sm_100a).
//
// Persistent CTAs of 256 threads walk (voxel tile, frame block) work items of
// one or more acquisitions.  A tile is tu x tv voxels across (the receive and
// the transmit-steering axes, one warp) by tz depths (one warp per depth);
// each thread owns one voxel and the FB frames of the block, and keeps its
// sums over receive elements and transmits in registers.
//
// For every (tx, rx) step the CTA stages the sample window its tile needs --
// rows [lo, lo + count) of the (tx, rx, frame block) slab, sample-major with
// the FB frames of a sample contiguous -- into shared memory as FP32 rows
// padded by 16 bytes (so the 16-byte loads of 8 consecutive rows hit
// distinct banks):
//   complex64 storage : cp.async 16-byte copies, three buffers, the copy of
//                       step s+2 in flight while step s computes;
//   FP16/BF16 storage : 16-byte register loads issued one step ahead and
//                       converted to FP32 once, when stored to the second of
//                       two buffers, so the inner loop never converts.
// The host sizes the buffers from an upper bound of every window of the
// acquisition (rcabf_geometry::window_rows) and picks a frame block that
// fits; a window beyond it is counted as an error and never read.
#pragma once

#include "das_common.cuh"

namespace rcabf {

template <int FB, int BYTES> struct ChunkT;   // register-staging chunk for FP16/BF16 slabs
template <int FB> struct ChunkT<FB, 16> { using T = uint4; };
template <int FB> struct ChunkT<FB, 8> { using T = uint2; };
template <int FB> struct ChunkT<FB, 4> { using T = uint32_t; };

constexpr int STAGE_REGS = 4;   // 16-byte chunks a thread may hold for one step

__device__ __forceinline__ float2 half2_bits_to_f2(uint32_t b, int store)
{
    if (store == ST_F16) {
        __half2 h;
        memcpy(&h, &b, 4);
        return __half22float2(h);
    }
    // bf16 -> f32 is a shift of the 16 bits into the high half
    return make_float2(__uint_as_float(b << 16), __uint_as_float(b & 0xffff0000u));
}

template <int MODE, int KIND, int FB, int STORE>
__global__ void __launch_bounds__(FUSED_THREADS)
fused_das_kernel(const __grid_constant__ FusedParams prm)
{
    using T = typename StoreT<STORE>::T;
    using KT = KindTraits<KIND>;
    constexpr bool TABLE = UsesTable<MODE, KIND>::value;
    constexpr bool ASYNC = (STORE == ST_F32);          // cp.async path
    constexpr int NST = ASYNC ? 3 : 2;                  // stage buffers
    constexpr int ES = (int)sizeof(T);
    constexpr int RAWB = FB * ES;                       // slab row bytes
    constexpr int SROWB = FB * 8;                       // staged (FP32) row bytes
    constexpr int CS = RAWB < 16 ? RAWB : 16;           // copy chunk
    constexpr int CPR = RAWB / CS;                      // chunks per row
    constexpr bool TWO_LEVEL = (MODE == MODE_REF);
    using Chunk = typename ChunkT<FB, CS>::T;

    extern __shared__ __align__(16) unsigned char smem[];
    const int tid = threadIdx.x;
    const int stride_s = prm.row_words * 4;
    const int stage_bytes = prm.wmax * stride_s;
    const int wt_bytes = TABLE ? WT_BYTES : 0;
    {
        // The launch must provide the table and NST window buffers; if it did
        // not, record the error and touch nothing (uniform across the block).
        unsigned dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (dyn < (unsigned)(wt_bytes + NST * stage_bytes) || stride_s < SROWB ||
            (!ASYNC && prm.wmax * CPR > STAGE_REGS * FUSED_THREADS) ||
            (TABLE && prm.jobs[0].g.wtab == nullptr)) {
            if (tid == 0) atomicAdd(prm.err_count, 1ull);
            return;
        }
    }
    float *wt = reinterpret_cast<float *>(smem);
    unsigned char *stages = smem + wt_bytes;
    if constexpr (TABLE) {
        // all jobs of a launch share the kernel kind, hence the table
        const float4 *src = reinterpret_cast<const float4 *>(prm.jobs[0].g.wtab);
        float4 *dst = reinterpret_cast<float4 *>(wt);
        for (int i = tid; i < WT_BYTES / 16; i += FUSED_THREADS) dst[i] = __ldg(src + i);
        __syncthreads();
    }

    for (int64_t item = blockIdx.x; item < prm.n_items; item += gridDim.x) {
        int ji = 0;
        while (ji + 1 < prm.n_jobs && prm.jobs[ji + 1].item_begin <= item) ++ji;
        const FusedJob &J = prm.jobs[ji];
        const DevGeom &g = J.g;
        const int lu = tid % J.tu;
        const int lv = (tid / J.tu) % J.tv;
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
        const int64_t iv = (int64_t)tv * J.tv + lv;
        const bool vox = iz < g.n_z && iu < g.n_u && iv < g.n_v;
        const int64_t rxkey = iu * g.n_z + iz;
        const int64_t txkey = iv * g.n_z + iz;
        const int64_t n_rxkey = g.n_u * g.n_z;
        const int64_t n_txkey = g.n_v * g.n_z;
        const int n_steps = g.n_tx * g.n_ele;
        const char *S = reinterpret_cast<const char *>(J.S);

        // acc: the voxel's sums; acc_tx: the current transmit's sum when the
        // transmits are added one by one (reference order), unused otherwise
        float2 acc[FB], acc_tx[FB];
#pragma unroll
        for (int f = 0; f < FB; ++f) { acc[f] = make_float2(0.f, 0.f); acc_tx[f] = acc[f]; }

        auto slab = [&](int tx, int rx) -> const char * {
            return S + (((int64_t)tx * g.n_ele + rx) * J.n_fb + fb) * J.slab_bytes;
        };
        auto window = [&](int s) -> Window {
            Window w;
            w.skip = true; w.lo = 0; w.count = 0; w.overflow = false;
            if (s >= n_steps) return w;
            const int tx = s / g.n_ele, rx = s % g.n_ele;
            return step_window<MODE, KIND>(J, tx, rx, tu, tv, tz, ab_value(g, tx, rx), prm.wmax);
        };
        // complex64 slabs: asynchronous copy of step s into buffer s % 3
        auto issue_async = [&](int s, const Window &w) {
            if (!w.skip && !w.overflow) {
                const char *src = slab(s / g.n_ele, s % g.n_ele) + (int64_t)w.lo * RAWB;
                unsigned char *dst = stages + (s % NST) * stage_bytes;
                const int nch = w.count * CPR;
                for (int c = tid; c < nch; c += FUSED_THREADS) {
                    const int r = c / CPR, q = c % CPR;
                    cp_async<CS>(dst + r * stride_s + q * CS, src + (int64_t)r * RAWB + q * CS);
                }
            }
            cp_async_commit();
        };
        // FP16/BF16 slabs: register loads of step s ...
        Chunk regs[STAGE_REGS];
        auto load_regs = [&](int s, const Window &w) {
            if (w.skip || w.overflow) return;
            const char *src = slab(s / g.n_ele, s % g.n_ele) + (int64_t)w.lo * RAWB;
            const int nch = w.count * CPR;
#pragma unroll
            for (int k = 0; k < STAGE_REGS; ++k) {
                const int c = tid + k * FUSED_THREADS;
                if (c < nch) regs[k] = __ldg(reinterpret_cast<const Chunk *>(src + (int64_t)c * CS));
            }
        };
        // ... converted to FP32 rows of buffer s % 2
        auto store_regs = [&](int s, const Window &w) {
            if (w.skip || w.overflow) return;
            unsigned char *dst = stages + (s % NST) * stage_bytes;
            const int nch = w.count * CPR;
#pragma unroll
            for (int k = 0; k < STAGE_REGS; ++k) {
                const int c = tid + k * FUSED_THREADS;
                if (c < nch) {
                    const int r = c / CPR, q = c % CPR;
                    float2 *o = reinterpret_cast<float2 *>(dst + r * stride_s + q * CS * 2);
                    uint32_t b[CS / 4];
                    memcpy(b, &regs[k], CS);
#pragma unroll
                    for (int v = 0; v < CS / 4; v += 2) {
                        if (v + 1 < CS / 4) {
                            const float2 x0 = half2_bits_to_f2(b[v], STORE), x1 = half2_bits_to_f2(b[v + 1], STORE);
                            *reinterpret_cast<float4 *>(o + v) = make_float4(x0.x, x0.y, x1.x, x1.y);
                        } else {
                            o[v] = half2_bits_to_f2(b[v], STORE);
                        }
                    }
                }
            }
        };

        // Prologue.
        Window wA = window(0), wB = window(1), wC;
        if constexpr (ASYNC) {
            issue_async(0, wA);
            issue_async(1, wB);
        } else {
            load_regs(0, wA);
            store_regs(0, wA);
            load_regs(1, wB);
            __syncthreads();
        }

        float4 tcur = make_float4(0.f, 0.f, 0.f, 0.f);
        bool cone_ok = true;
        float4 enext = vox ? __ldg(&g.rx_tab[rxkey]) : make_float4(0.f, 0.f, 0.f, 0.f);

        for (int s = 0; s < n_steps; ++s) {
            const int tx = s / g.n_ele, rx = s % g.n_ele;
            if constexpr (ASYNC) {
                cp_async_wait<NST - 2>();
                __syncthreads();                   // step s landed; step s-1's buffer is free
                wC = window(s + 2);
                issue_async(s + 2, wC);
            }

            const float4 e = enext;
            if (vox && s + 1 < n_steps) {
                const int rx1 = (s + 1) % g.n_ele;
                enext = __ldg(&g.rx_tab[(int64_t)rx1 * n_rxkey + rxkey]);
            }
            if (rx == 0 && vox) {
                tcur = __ldg(&g.tx_tab[(int64_t)tx * n_txkey + txkey]);
                const float cv = (MODE == MODE_EXACT) ? tcur.w : tcur.y;
                cone_ok = cv != 0.0f;
                if (g.cone_u != nullptr) cone_ok = cone_ok && g.cone_u[(int64_t)tx * n_rxkey + rxkey] != 0;
            }

            if (!wA.skip && vox && cone_ok) {
                const float ab = ab_value(g, tx, rx);
                Setup<KIND> st;
                if constexpr (MODE == MODE_EXACT)
                    setup_exact<KIND>(tcur, e, ab, ab_phasor(g, tx, rx), J.n_sample, st, TABLE ? wt : nullptr);
                else
                    setup_ref<KIND>(tcur, e, ab, g.ref, J.n_sample, st);
                if (st.ok) {
                    const int row0 = st.n0 - KT::LO - wA.lo;
                    float2 (&a)[FB] = TWO_LEVEL ? acc_tx : acc;
                    if (row0 < 0 || row0 + KT::TAPS > wA.count || wA.overflow) {
                        // never expected: the host sizes wmax from an upper bound
                        // of every window; record the violation, skip the taps
                        atomicAdd(prm.err_count, 1ull);
                    } else {
                        const char *rowp = reinterpret_cast<const char *>(stages) +
                                           (s % NST) * stage_bytes + row0 * stride_s;
                        frame_loop<MODE, KIND, FB, ST_F32>(rowp, stride_s, st, a);
                    }
                }
            }

            if (rx == g.n_ele - 1) {  // end of a transmit
                float2 (&src)[FB] = TWO_LEVEL ? acc_tx : acc;
                if (!J.compound && vox) {
                    const int64_t pix = iz * g.s_z + iu * g.s_u + iv * g.s_v;
#pragma unroll
                    for (int f = 0; f < FB; ++f) {
                        const int fr = fb * FB + f;
                        if (fr < J.n_frame) {
                            float2 *o = J.out + ((int64_t)fr * g.n_tx + tx) * g.n_pix + pix;
                            if (J.accumulate) { float2 v = *o; v.x += src[f].x; v.y += src[f].y; *o = v; }
                            else *o = src[f];
                        }
                    }
                }
                if (!J.compound) {
#pragma unroll
                    for (int f = 0; f < FB; ++f) src[f] = make_float2(0.f, 0.f);
                } else if constexpr (TWO_LEVEL) {
#pragma unroll
                    for (int f = 0; f < FB; ++f) {
                        acc[f].x = __fadd_rn(acc[f].x, src[f].x);
                        acc[f].y = __fadd_rn(acc[f].y, src[f].y);
                        src[f] = make_float2(0.f, 0.f);
                    }
                }
            }

            if constexpr (!ASYNC) {
                store_regs(s + 1, wB);             // buffer (s+1)%2 was last read by step s-1
                wC = window(s + 2);
                load_regs(s + 2, wC);
                __syncthreads();                   // step s+1 staged; step s reads done
            }
            wA = wB;
            wB = wC;
        }
        if constexpr (ASYNC) cp_async_wait<0>();
        __syncthreads();  // all buffers idle before the next work item reuses them

        if (J.compound && vox) {
            const int64_t pix = iz * g.s_z + iu * g.s_u + iv * g.s_v;
#pragma unroll
            for (int f = 0; f < FB; ++f) {
                const int fr = fb * FB + f;
                if (fr < J.n_frame) {
                    float2 *o = J.out + (int64_t)fr * g.n_pix + pix;
                    if (J.accumulate) { float2 v = *o; v.x += acc[f].x; v.y += acc[f].y; *o = v; }
                    else *o = acc[f];
                }
            }
        }
    }
}

}  // namespace rcabf
