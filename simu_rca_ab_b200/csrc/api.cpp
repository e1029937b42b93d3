// C ABI of librcabf (include/rcabf.h): geometry handles, launch planning and
// the beamform entry points.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/rcabf.h"
#include "geometry.h"
#include "launchers.h"
#include "plan.h"

using namespace rcabf;

namespace rcabf {

std::atomic<int64_t> g_launches{0};

// Detail of the last RCABF_ERR_CUDA of this thread (rcabf_last_error()).
static thread_local char g_last_err[256] = "";

static int cuda_fail(cudaError_t e, const char *where)
{
    snprintf(g_last_err, sizeof(g_last_err), "%s: %s (cudaError %d)", where, cudaGetErrorString(e), (int)e);
    return RCABF_ERR_CUDA;
}

struct DeviceState {
    unsigned long long *err = nullptr;
    int n_sm = 0;
    std::mutex mu;
    std::map<std::array<int64_t, 5>, int> occ;        // (variant..., smem) -> CTAs/SM
    // The dynamic shared-memory limit is an attribute of the kernel function,
    // so it is only ever raised: variant -> largest limit set so far.
    std::map<std::array<int64_t, 4>, size_t> smem_limit;
};

static std::mutex g_dev_mu;
static std::map<int, DeviceState *> g_dev;

// with_err: also allocate the device error counter if it does not exist yet
// (rcabf_beamform_noalloc asks for the host-side state only).
DeviceState *device_state(int dev, bool with_err = true)
{
    std::lock_guard<std::mutex> lk(g_dev_mu);
    auto it = g_dev.find(dev);
    DeviceState *s;
    if (it != g_dev.end()) {
        s = it->second;
    } else {
        s = new DeviceState();
        cudaDeviceGetAttribute(&s->n_sm, cudaDevAttrMultiProcessorCount, dev);
        g_dev[dev] = s;
    }
    if (with_err && !s->err) {
        if (cudaMalloc(&s->err, sizeof(unsigned long long)) != cudaSuccess) s->err = nullptr;
        else cudaMemset(s->err, 0, sizeof(unsigned long long));
    }
    return s;
}

unsigned long long *current_error_counter()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
    return device_state(dev)->err;
}

void count_launches(int64_t n) { g_launches += n; }

static int pow2_ceil(int64_t x)
{
    int p = 1;
    while (p < x && p < (1 << 30)) p <<= 1;
    return p;
}

TileShape default_tile(const rcabf_geometry *g)
{
    // Lanes of a warp cover a (u, v) patch at one depth: receive and transmit
    // delays differ little across it, so the taps of a warp fall on few rows
    // of the shared-memory window.  Warps stack along z.
    int tu = std::min(4, pow2_ceil(g->n_u));
    int tv = std::min(8, pow2_ceil(g->n_v));
    if (tu * tv < 32 && g->n_u > tu) tu = std::min(32 / tv, pow2_ceil(g->n_u));
    const int tz = FUSED_THREADS / (tu * tv);
    return TileShape{tu, tv, tz};
}

bool fb_supported(int mode, int fb)
{
    switch (fb) {
    case 1: case 2: case 4: case 8: case 16: return true;
    case 24: case 32: case 40: return mode == MODE_EXACT;
    default: return false;
    }
}

// Rows one staging buffer can hold at frame block fb.
static int stage_capacity_rows(const rcabf_geometry *g, int store, int fb)
{
    const size_t tbl = fused_table_bytes(g->mode, g->kind);
    const int cap = (int)((SMEM_BUDGET - tbl) / ((size_t)fused_stages(store) * fused_row_words(fb) * 4));
    return std::min(cap, fused_stage_rows_cap(store, fb));
}

// Frame block: each block repeats the per-(voxel, rx, tx) setup, worth about
// SETUP_FRAMES frames of work, and pads the last block; pick the block that
// minimises blocks x (FB + SETUP_FRAMES) among the compiled sizes whose
// staging buffers hold the largest window (`need` rows).  0 = none fits.
int choose_fb(const rcabf_geometry *g, int store, int64_t n_frame, int requested, int need)
{
    const int cands[] = {1, 2, 4, 8, 16, 24, 32, 40};
    const double SETUP_FRAMES = 4.0;
    int best = 0;
    double best_cost = 1e300;
    for (int fb : cands) {
        if (!fb_supported(g->mode, fb)) continue;
        if (requested > 0 && fb > requested) continue;
        if (requested <= 0 && fb > 2 * n_frame && fb > 1) continue;
        if (stage_capacity_rows(g, store, fb) < need) continue;
        const double blocks = (double)((n_frame + fb - 1) / fb);
        const double cost = requested > 0 ? -fb : blocks * (fb + SETUP_FRAMES);
        if (cost < best_cost - 1e-9) { best_cost = cost; best = fb; }
    }
    return best;
}

int plan_beamform(rcabf_geometry *g, const rcabf_beamform_args *a, Plan &p, const TuneChoice *force)
{
    if (!g || !a) return RCABF_ERR_INVALID_ARGUMENT;
    if (a->struct_size != (int32_t)sizeof(rcabf_beamform_args)) return RCABF_ERR_INVALID_ARGUMENT;
    if (a->n_sample < 1 || a->n_frame < 1) return RCABF_ERR_SHAPE_MISMATCH;
    if (a->n_ch != g->n_ele || a->n_tx != g->n_tx) return RCABF_ERR_SHAPE_MISMATCH;
    if (a->n_sample > (1 << 24) || a->n_frame > (1 << 24)) return RCABF_ERR_UNSUPPORTED;
    if (a->iq_dtype < RCABF_IQ_C64 || a->iq_dtype > RCABF_IQ_RF_F32) return RCABF_ERR_INVALID_ARGUMENT;
    if (a->storage < RCABF_STORE_F32 || a->storage > RCABF_STORE_BF16) return RCABF_ERR_INVALID_ARGUMENT;
    if (g->mode == MODE_REF && a->storage != RCABF_STORE_F32) return RCABF_ERR_UNSUPPORTED;
    const int fb_req = a->frames_per_block;
    const bool tc_req = a->kernel == RCABF_KERNEL_FUSED_TC || a->kernel == RCABF_KERNEL_FUSED_TC_FP16W;
    if (fb_req != 0 && !tc_req && !fb_supported(g->mode, fb_req)) return RCABF_ERR_INVALID_ARGUMENT;
    if (a->per_channel && a->compound) return RCABF_ERR_INVALID_ARGUMENT;   // no sum over elements: none over tx
    if (a->kernel < RCABF_KERNEL_AUTO || a->kernel > RCABF_KERNEL_FUSED_TC_FP16W) return RCABF_ERR_INVALID_ARGUMENT;
    p = Plan{};
    p.kernel = (a->kernel == RCABF_KERNEL_PLAIN || a->per_channel) ? RCABF_KERNEL_PLAIN : RCABF_KERNEL_FUSED;
    if (p.kernel == RCABF_KERNEL_PLAIN) {
        // per-channel output: all frames in one launch unless the
        // one-launch-per-frame kernel is asked for by name
        p.pc_all = a->per_channel && a->kernel != RCABF_KERNEL_PLAIN ? 1 : 0;
        p.total = 0;
        return RCABF_OK;
    }
    p.store = a->storage;
    const int es = store_bytes(p.store);
    TuneChoice tuned;
    if (!force) {   // a choice the autotuner measured for this geometry, frames and storage
        std::lock_guard<std::mutex> lk(g->mu);
        auto it = g->tuned.find({a->n_frame, (int64_t)a->storage});
        const int vb_req = a->kernel == RCABF_KERNEL_FUSED_TMEM ? 2 : a->kernel == RCABF_KERNEL_FUSED_REGS ? 1 : -1;
        if (it != g->tuned.end() && !tc_req && (fb_req == 0 || fb_req == it->second.fb) &&
            !((it->second.vb || it->second.tc) && a->kernel == RCABF_KERNEL_FUSED_NOBLOCK) &&
            !(it->second.tc && (vb_req >= 0 || !a->compound)) && (vb_req < 0 || vb_req == it->second.vb)) {
            tuned = it->second;
            force = &tuned;
        }
    }
    auto layout = [&](int tile_v_extent) {
        p.n_fb = (int)((a->n_frame + p.fb - 1) / p.fb);
        p.tiles_z = (int)((g->n_z + p.ts.tz - 1) / p.ts.tz);
        p.tiles_u = (int)((g->n_u + p.ts.tu - 1) / p.ts.tu);
        p.tiles_v = (int)((g->n_v + tile_v_extent - 1) / tile_v_extent);
        p.row_words = fused_row_words(p.fb);
        p.slab_bytes = ((int64_t)(p.tc ? p.tc_rows : a->n_sample) * p.fb * es + 15) / 16 * 16;
        auto al = [](size_t x) { return (x + 255) / 256 * 256; };
        size_t off = 0;
        p.off_S = off;
        // (tensor-core plans: the slabs, then right after them the same
        // slabs holding (-im, re), one row range of the kernel's tensor map)
        off += al((size_t)g->n_tx * g->n_ele * p.n_fb * p.slab_bytes * (p.tc ? 2 : 1));
        p.off_rxr = off;
        off += al((size_t)g->n_ele * p.tiles_u * p.tiles_z * sizeof(float2));
        p.off_txr = off;
        off += al((size_t)g->n_tx * p.tiles_v * p.tiles_z * sizeof(float2));
        p.total = off;
        p.n_items = (int64_t)p.n_fb * p.tiles_z * p.tiles_u * p.tiles_v;
    };

    // Tensor-core kernel: FP16 slabs (BF16 slabs with hi + remainder weights),
    // exact tables, compounded output, a
    // rectilinear grid whose 4 x 32 x 1 tiles need windows of at most 32
    // rows, at least 32 frames; frame blocks of a multiple of 8 frames, as
    // few as the tensor-memory budget allows (the weights are built once
    // per block).
    // The planner's own choice (kernel AUTO / FUSED, no frame block asked
    // for) takes it, with hi + remainder weights, where it applies to 32
    // frames or more; by name or by a stored / forced choice it also takes
    // fewer frames (one padded block).
    const int named_tc = force ? force->tc
                         : a->kernel == RCABF_KERNEL_FUSED_TC       ? 2
                         : a->kernel == RCABF_KERNEL_FUSED_TC_FP16W ? 1
                                                                    : 0;
    const bool auto_tc = !named_tc && !force && fb_req == 0 &&
                         (a->kernel == RCABF_KERNEL_AUTO || a->kernel == RCABF_KERNEL_FUSED) && a->n_frame >= 32;
    const int want_tc = named_tc ? named_tc : auto_tc ? 2 : 0;
    if (want_tc) {
        const int fbmax = tc_max_frames_per_block(want_tc == 2);
        const bool store_ok = a->storage == RCABF_STORE_F16 || (a->storage == RCABF_STORE_BF16 && want_tc == 2);
        bool ok = g->mode == MODE_EXACT && store_ok && a->compound && !a->per_channel &&
                  g->grid_kind == RCABF_GRID_RECTILINEAR && a->n_sample >= 2;
        // the 128-voxel tile whose windows are shortest (a forced shape if given)
        TileShape tts{TC_TILE_U, TC_TILE_V, 1};
        if (ok) {
            int best_rows = 1 << 30;
            const TileShape shapes[] = {{4, 32, 1}, {8, 16, 1}, {2, 64, 1}, {16, 8, 1}, {1, 128, 1}, {32, 4, 1}};
            for (const TileShape &t : shapes) {
                if (force && force->ts.tu > 0 && (t.tu != force->ts.tu || t.tv != force->ts.tv)) continue;
                const int rows = g->window_rows(t);
                if (rows < best_rows) { best_rows = rows; tts = t; }
            }
            ok = best_rows <= TC_MAX_ROWS;
        }
        int fb = 0;
        if (ok) {
            const int64_t nfb = (a->n_frame + fbmax - 1) / fbmax;
            fb = std::max<int>(32, (int)(((a->n_frame + nfb - 1) / nfb + 7) / 8 * 8));
            if (force && force->fb) fb = force->fb;
            else if (fb_req > 0) fb = fb_req;
            ok = fb >= 32 && fb <= fbmax && fb % 8 == 0;
        }
        if (ok) {
            p.tc = want_tc;
            p.fb = fb;
            p.ts = tts;
            p.tc_rows = (int)a->n_sample + TC_MAX_ROWS;
            layout(tts.tv);
            ok = 2 * (int64_t)g->n_tx * g->n_ele * p.n_fb * p.tc_rows < ((int64_t)1 << 31);
        }
        if (ok) {
            p.wmax = TC_MAX_ROWS;
            p.smem = tc_launch_smem(fb);
            return RCABF_OK;
        }
        p = Plan{};
        if (named_tc) return RCABF_ERR_UNSUPPORTED;
        p.kernel = RCABF_KERNEL_FUSED;   // not tensor-core work: the SIMT kernels below
        p.store = a->storage;
    }

    // Voxel-blocked kernel: exact tables, a steering axis to block along,
    // frames in pairs, and at most 2 rows of shift inside a block.  Its
    // accumulators live in registers (vb = 1) or, for frame blocks of 8 and
    // 16, in tensor memory (vb = 2).
    const int want_vb = force ? force->vb
                        : a->kernel == RCABF_KERNEL_FUSED_TMEM ? 2
                        : a->kernel == RCABF_KERNEL_FUSED_REGS ? 1
                                                               : 0;   // 0: the planner's choice
    const bool vb_fb_ok = force ? force->vb >= 1
                                : fb_req == 0 ? a->n_frame >= 2
                                              : (fb_req == 2 || fb_req == 4 || fb_req == 8 || fb_req == 16);
    if (g->mode == MODE_EXACT && vb_fb_ok && a->kernel != RCABF_KERNEL_FUSED_NOBLOCK) {
        const int d = g->vb_shift(VB_BLOCK);
        if (d >= 1 && d <= 2) {
            const int tu = std::min(4, pow2_ceil(g->n_u));
            const int tvb = 2;
            TileShape vts{tu, tvb, VB_THREADS_HOST / (tu * tvb)};
            if (force) {
                if (force->ts.tu * force->ts.tv * force->ts.tz != VB_THREADS_HOST) return RCABF_ERR_UNSUPPORTED;
                vts = force->ts;
            }
            const int need = (int)std::min<int64_t>(
                g->window_rows(TileShape{vts.tu, vts.tv * VB_BLOCK, vts.tz}) + d, a->n_sample);
            auto pick_fb = [&](int tm) {   // the largest frame block whose window fits
                for (int c : {16, 8, 4, 2}) {
                    if (force && c != force->fb) continue;
                    if (!force && fb_req > 0 && c != fb_req) continue;
                    // the planner's choice: at most the frame count rounded up to a
                    // power of two (a block more than half empty costs more than
                    // the setup it saves: per item t ~ setup + FB x frame cost,
                    // setup ~ 13 frames); a store asked for by name may pad to 2x
                    const int64_t lim = want_vb ? 2 * a->n_frame : pow2_ceil(a->n_frame);
                    if (!force && fb_req == 0 && c > lim) continue;
                    const int cap = std::min<int>((int)(VB_SMEM_BUDGET / ((size_t)fused_stages(p.store) *
                                                                           fused_row_words(c) * 4)),
                                                  vb_stage_rows_cap(p.store, c));
                    if (cap >= need) return c;
                }
                return 0;
            };
            int tm = want_vb == 2 ? 1 : want_vb == 1 ? 0 : VB_TMEM_DEFAULT;
            int fb = pick_fb(tm);
            if (!fb && tm && want_vb == 0) fb = pick_fb(tm = 0);   // blocks below 8 frames: registers
            if (fb) {
                p.vb = tm ? 2 : 1;
                p.d = d;
                p.fb = fb;
                p.ts = vts;
                layout(vts.tv * VB_BLOCK);
                p.wmax = need;
                p.smem = vb_smem_bytes(p.store, p.wmax, p.row_words, tm ? kind_taps(g->kind) + d : 0);
                return RCABF_OK;
            }
        }
    }
    if (want_vb) return RCABF_ERR_UNSUPPORTED;

    p.ts = default_tile(g);
    if (force && force->ts.tu > 0) {
        if (force->ts.tu * force->ts.tv * force->ts.tz != FUSED_THREADS) return RCABF_ERR_UNSUPPORTED;
        p.ts = force->ts;
    }
    // the largest window of any (tile, tx, rx) step, rounded up: the staging
    // buffers hold it, so the kernel never needs a fallback path
    const int need = std::min<int64_t>(g->window_rows(p.ts), a->n_sample);
    p.fb = choose_fb(g, p.store, a->n_frame, force ? force->fb : fb_req, need);
    if (force && p.fb != force->fb) return RCABF_ERR_UNSUPPORTED;
    if (p.fb == 0) {  // no staging buffer holds the window: one-frame kernel
        p.kernel = RCABF_KERNEL_PLAIN;
        p.total = 0;
        return RCABF_OK;
    }
    layout(p.ts.tv);
    p.wmax = std::max(kind_taps(g->kind), need);
    p.smem = fused_smem_bytes(g->mode, g->kind, p.store, p.wmax, p.row_words);
    return RCABF_OK;
}

static void mark(const rcabf_beamform_args *a, int i, cudaStream_t st)
{
    if (a->stage_events && a->stage_events[i]) cudaEventRecord((cudaEvent_t)a->stage_events[i], st);
}

// Fills the per-job descriptor and launches the job's ingest and range kernels.
int stage_job(rcabf_geometry *g, const rcabf_beamform_args *a, const Plan &p, FusedJob &J, cudaStream_t st,
              const rcabf_beamform_args *marks = nullptr)
{
    char *ws = reinterpret_cast<char *>(a->workspace);
    IngestParams ip{};
    ip.iq = a->iq; ip.iq_dtype = a->iq_dtype; ip.n_sample = (int)a->n_sample; ip.n_ele = g->n_ele;
    ip.n_tx = g->n_tx; ip.n_frame = a->n_frame; ip.fb = p.fb; ip.n_fb = p.n_fb;
    ip.S = ws + p.off_S; ip.slab_bytes = p.slab_bytes; ip.n_rows = p.tc ? p.tc_rows : 0;
    ip.S2 = p.tc ? ws + p.off_S + (size_t)g->n_tx * g->n_ele * p.n_fb * p.slab_bytes : nullptr;
    cudaError_t ce = launch_ingest(ip, p.store, st);
    if (ce != cudaSuccess) return cuda_fail(ce, "ingest launch");
    if (marks) mark(marks, 1, st);
    RangeParams rr{};
    rr.tab = g->rx_tab; rr.out = reinterpret_cast<float2 *>(ws + p.off_rxr); rr.rows = g->n_ele;
    rr.n_a = g->n_u; rr.n_z = g->n_z; rr.ta = p.ts.tu; rr.tz = p.ts.tz; rr.tiles_a = p.tiles_u;
    rr.tiles_z = p.tiles_z; rr.mode = g->mode; rr.is_rx = 1;
    if ((ce = launch_range(rr, st)) != cudaSuccess) return cuda_fail(ce, "rx range launch");
    RangeParams tr = rr;
    tr.tab = g->tx_tab; tr.out = reinterpret_cast<float2 *>(ws + p.off_txr); tr.rows = g->n_tx;
    tr.n_a = g->n_v; tr.ta = p.vb ? p.ts.tv * VB_BLOCK : p.ts.tv; tr.tiles_a = p.tiles_v; tr.is_rx = 0;
    if ((ce = launch_range(tr, st)) != cudaSuccess) return cuda_fail(ce, "tx range launch");
    g_launches += 3;
    if (marks) mark(marks, 2, st);

    J = FusedJob{};
    J.g = g->dev();
    J.S = ws + p.off_S;
    J.slab_bytes = p.slab_bytes;
    J.rx_range = reinterpret_cast<const float2 *>(ws + p.off_rxr);
    J.tx_range = reinterpret_cast<const float2 *>(ws + p.off_txr);
    J.out = reinterpret_cast<float2 *>(a->out);
    J.n_fb = p.n_fb; J.n_frame = (int)a->n_frame; J.n_sample = (int)a->n_sample;
    J.compound = a->compound ? 1 : 0; J.accumulate = a->accumulate ? 1 : 0;
    J.tiles_z = p.tiles_z; J.tiles_u = p.tiles_u; J.tiles_v = p.tiles_v;
    J.tu = p.ts.tu; J.tv = p.ts.tv; J.tz = p.ts.tz;
    return RCABF_OK;
}

// Resident CTAs per SM of the plan's fused kernel at `smem` bytes of dynamic
// shared memory (sets the kernel's shared-memory limit on first use).
static int resident_ctas(const rcabf_geometry *g0, const Plan &p, size_t smem, DeviceState *ds, int &occ)
{
    // variant: (mode, or 2 vb + row shift for the voxel-blocked kernels; kind; fb; store)
    const std::array<int64_t, 4> var{p.vb ? 2 * p.vb + p.d : g0->mode, g0->kind, p.fb, p.store};
    const std::array<int64_t, 5> key{var[0], var[1], var[2], var[3], (int64_t)smem};
    std::lock_guard<std::mutex> lk(ds->mu);
    auto lim = ds->smem_limit.find(var);
    if (lim == ds->smem_limit.end() || lim->second < smem) {
        const cudaError_t pe = p.vb ? prepare_fused_vb(g0->kind, p.d, p.vb == 2, p.fb, p.store, smem)
                                    : prepare_fused(g0->mode, g0->kind, p.fb, p.store, smem);
        if (pe != cudaSuccess) return cuda_fail(pe, "fused kernel shared-memory attribute");
        ds->smem_limit[var] = smem;
    }
    auto oc = ds->occ.find(key);
    if (oc == ds->occ.end()) {
        const int o = p.vb ? fused_vb_occupancy(g0->kind, p.d, p.vb == 2, p.fb, p.store, smem)
                           : fused_occupancy(g0->mode, g0->kind, p.fb, p.store, smem);
        oc = ds->occ.emplace(key, o).first;
    }
    occ = std::max(1, oc->second);
    return RCABF_OK;
}

int launch_fused_jobs(rcabf_geometry *g0, FusedParams &prm, const Plan &p, cudaStream_t st)
{
    // a counter set by the caller (rcabf_beamform_noalloc) is kept
    DeviceState *ds = device_state(g0->device, prm.err_count == nullptr);
    if (!prm.err_count) prm.err_count = ds->err;
    if (p.tc) {   // one launch per job (a persistent grid of one CTA per SM each)
        for (int j = 0; j < prm.n_jobs; ++j) {
            const int64_t end = j + 1 < prm.n_jobs ? prm.jobs[j + 1].item_begin : prm.n_items;
            const cudaError_t le = launch_fused_tc(g0->kind, p.tc == 2, p.store == ST_BF16, prm.jobs[j], p.fb, p.tc_rows,
                                                   end - prm.jobs[j].item_begin, prm.err_count, ds->n_sm, st);
            if (le != cudaSuccess) return cuda_fail(le, "tensor-core kernel launch");
            g_launches += 1;
        }
        return RCABF_OK;
    }
    const size_t smem = p.vb ? vb_smem_bytes(p.store, prm.wmax, prm.row_words,
                                             p.vb == 2 ? kind_taps(g0->kind) + p.d : 0)
                             : fused_smem_bytes(g0->mode, g0->kind, p.store, prm.wmax, prm.row_words);
    int occ = 0;
    const int so = resident_ctas(g0, p, smem, ds, occ);
    if (so != RCABF_OK) return so;
    const int64_t grid = std::min<int64_t>(prm.n_items, (int64_t)ds->n_sm * occ);
    if (grid <= 0) return RCABF_OK;
    const cudaError_t le = p.vb ? launch_fused_vb(g0->kind, p.d, p.vb == 2, p.fb, p.store, prm, (int)grid, smem, st)
                                : launch_fused(g0->mode, g0->kind, p.fb, p.store, prm, (int)grid, smem, st);
    if (le != cudaSuccess) return cuda_fail(le, "fused kernel launch");
    g_launches += 1;
    return RCABF_OK;
}

static int check_ptrs(const rcabf_beamform_args *a, const Plan &p)
{
    if (!a->iq || !a->out) return RCABF_ERR_INVALID_ARGUMENT;
    if (p.kernel == RCABF_KERNEL_FUSED) {
        if (a->workspace_bytes < p.total || (p.total && !a->workspace)) return RCABF_ERR_WORKSPACE_TOO_SMALL;
        if (((uintptr_t)a->workspace) % 256) return RCABF_ERR_INVALID_ARGUMENT;
    }
    if (((uintptr_t)a->out) % 8) return RCABF_ERR_INVALID_ARGUMENT;
    return RCABF_OK;
}

static int beamform_planned(rcabf_geometry *g, const rcabf_beamform_args *a, const Plan &p, cudaStream_t st);

int beamform_one(rcabf_geometry *g, const rcabf_beamform_args *a, cudaStream_t st)
{
    Plan p;
    int s = plan_beamform(g, a, p);
    if (s != RCABF_OK) return s;
    return beamform_planned(g, a, p, st);
}

// One beamform call with a given plan (the autotuner's candidates).
static int beamform_planned(rcabf_geometry *g, const rcabf_beamform_args *a, const Plan &p, cudaStream_t st)
{
    int s;
    if ((s = check_ptrs(a, p)) != RCABF_OK) return s;
    device_state(g->device);
    mark(a, 0, st);
    if (p.kernel == RCABF_KERNEL_PLAIN) {
        mark(a, 1, st);
        mark(a, 2, st);
        PlainParams pp{};
        pp.g = g->dev(); pp.iq = a->iq; pp.iq_dtype = a->iq_dtype; pp.n_sample = (int)a->n_sample;
        pp.n_frame = a->n_frame; pp.compound = a->compound ? 1 : 0; pp.accumulate = a->accumulate ? 1 : 0;
        pp.per_channel = a->per_channel ? 1 : 0;
        pp.out = reinterpret_cast<float2 *>(a->out);
        pp.err_count = device_state(g->device)->err;
        if (p.pc_all) {
            pp.frame = -1;   // every frame
            const cudaError_t le = launch_plain(g->mode, g->kind, pp, st);
            if (le != cudaSuccess) return cuda_fail(le, "per-channel kernel launch");
            g_launches += 1;
        }
        for (int64_t f = 0; f < a->n_frame && !p.pc_all; ++f) {
            pp.frame = f;
            const cudaError_t le = launch_plain(g->mode, g->kind, pp, st);
            if (le != cudaSuccess) return cuda_fail(le, "plain kernel launch");
            g_launches += 1;
        }
    } else {
        FusedParams prm{};
        if ((s = stage_job(g, a, p, prm.jobs[0], st, a)) != RCABF_OK) return s;
        prm.jobs[0].item_begin = 0;
        prm.n_jobs = 1;
        prm.wmax = p.wmax;
        prm.row_words = p.row_words;
        prm.n_items = p.n_items;
        if ((s = launch_fused_jobs(g, prm, p, st)) != RCABF_OK) return s;
    }
    mark(a, 3, st);
    if (a->mask) {
        const cudaError_t me = launch_mask(g->dev(), a->mask, a->compound ? 1 : 0, a->accumulate ? 1 : 0, st);
        if (me != cudaSuccess) return cuda_fail(me, "mask kernel launch");
        g_launches += 1;
    }
    mark(a, 4, st);
    return RCABF_OK;
}

// Static workspace of rcabf_beamform_noalloc, per device: looked up once with
// the device current, its error counter cleared then.  Every call checks that
// the geometry's device is the current one before it uses the cached
// addresses: they are device addresses of that GPU only.
struct NoallocRegion {
    void *ws = nullptr;
    unsigned long long *err = nullptr;
};
static std::mutex g_noalloc_mu;
static std::map<int, NoallocRegion> g_noalloc;

static int noalloc_setup(int dev, NoallocRegion &r, bool create)
{
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return cuda_fail(e, "noalloc: cudaGetDevice");
    if (cur != dev) {
        snprintf(g_last_err, sizeof(g_last_err),
                 "noalloc: the geometry's device %d is not the current device %d", dev, cur);
        return RCABF_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    auto it = g_noalloc.find(dev);
    if (it != g_noalloc.end()) { r = it->second; return RCABF_OK; }
    if (!create) return RCABF_ERR_PENDING;
    NoallocRegion n;
    if ((e = noalloc_region(&n.ws, &n.err)) != cudaSuccess) return cuda_fail(e, "noalloc set-up: cudaGetSymbolAddress");
    if ((e = cudaMemset(n.err, 0, sizeof(unsigned long long))) != cudaSuccess)
        return cuda_fail(e, "noalloc set-up: clearing the error counter");
    g_noalloc[dev] = n;
    r = n;
    return RCABF_OK;
}

int beamform_noalloc(rcabf_geometry *g, const rcabf_beamform_args *a, cudaStream_t st)
{
    if (!a) return RCABF_ERR_INVALID_ARGUMENT;
    Plan p;
    int s = plan_beamform(g, a, p);
    if (s != RCABF_OK) return s;
    if (p.kernel != RCABF_KERNEL_FUSED) {
        snprintf(g_last_err, sizeof(g_last_err), "noalloc: the plan is the plain kernel; this entry runs the fused kernel only");
        return RCABF_ERR_UNSUPPORTED;
    }
    if (p.total > RCABF_NOALLOC_WORKSPACE_BYTES) {
        snprintf(g_last_err, sizeof(g_last_err),
                 "noalloc: the plan needs %zu workspace bytes; the static workspace holds %zu", p.total,
                 (size_t)RCABF_NOALLOC_WORKSPACE_BYTES);
        return RCABF_ERR_WORKSPACE_TOO_SMALL;
    }
    NoallocRegion r;
    if ((s = noalloc_setup(g->device, r, true)) != RCABF_OK) return s;
    rcabf_beamform_args b = *a;
    b.workspace = r.ws;
    b.workspace_bytes = RCABF_NOALLOC_WORKSPACE_BYTES;
    if ((s = check_ptrs(&b, p)) != RCABF_OK) return s;
    mark(&b, 0, st);
    FusedParams prm{};
    if ((s = stage_job(g, &b, p, prm.jobs[0], st, &b)) != RCABF_OK) return s;
    prm.jobs[0].item_begin = 0;
    prm.n_jobs = 1;
    prm.wmax = p.wmax;
    prm.row_words = p.row_words;
    prm.n_items = p.n_items;
    prm.err_count = r.err;
    if ((s = launch_fused_jobs(g, prm, p, st)) != RCABF_OK) return s;
    mark(&b, 3, st);
    if (b.mask) {
        const cudaError_t me = launch_mask(g->dev(), b.mask, b.compound ? 1 : 0, b.accumulate ? 1 : 0, st);
        if (me != cudaSuccess) return cuda_fail(me, "mask kernel launch");
        g_launches += 1;
    }
    mark(&b, 4, st);
    return RCABF_OK;
}

}  // namespace rcabf

// --------------------------------------------------------------------------
// C ABI
// --------------------------------------------------------------------------
extern "C" {

const char *rcabf_status_string(int s)
{
    switch (s) {
    case RCABF_OK: return "ok";
    case RCABF_ERR_DATA_NOT_NUMERIC: return "bfVirtualSourceGeneric_RCA:dataNotNumeric";
    case RCABF_ERR_OPTIONS_NOT_STRUCT: return "bfVirtualSourceGeneric_RCA:OptionsNotStruct";
    case RCABF_ERR_INTERPOLATION_INVALID: return "bfVirtualSourceGeneric_RCA:flagInterpolationLanczosInvalid";
    case RCABF_ERR_COMPOUNDING_INVALID: return "bfVirtualSourceGeneric_RCA:flagCompoundingInvalid";
    case RCABF_ERR_MASK_TRANSMIT_INVALID: return "bfVirtualSourceGeneric_RCA:flagMaskTransmitInvalid";
    case RCABF_ERR_DECREASE_FACTOR_INVALID: return "bfVirtualSourceGeneric_RCA:decreaseFactorGPUInvalid";
    case RCABF_ERR_GRID_MISSING: return "bfVirtualSourceGeneric_RCA:gridBfMissing";
    case RCABF_ERR_GRID_INVALID: return "bfVirtualSourceGeneric_RCA:gridBfInvalid";
    case RCABF_ERR_POS_ELE_MISSING: return "bfVirtualSourceGeneric_RCA:posEleMissing";
    case RCABF_ERR_POS_ELE_INVALID: return "bfVirtualSourceGeneric_RCA:posEleInvalid";
    case RCABF_ERR_APERTURE_X_INVALID: return "bfVirtualSourceGeneric_RCA:apertureXInvalid";
    case RCABF_ERR_APERTURE_Y_INVALID: return "bfVirtualSourceGeneric_RCA:apertureYInvalid";
    case RCABF_ERR_APERTURE_Z_INVALID: return "bfVirtualSourceGeneric_RCA:apertureZInvalid";
    case RCABF_ERR_TRANSMIT_NOT_STRUCT: return "bfVirtualSourceGeneric_RCA:TransmitNotStruct";
    case RCABF_ERR_THETA_OR_VS_REQUIRED: return "bfVirtualSourceGeneric_RCA:ThetaORVirtualSourceRequired";
    case RCABF_ERR_TILTS_NOT_SAME_LENGTH: return "bfVirtualSourceGeneric_RCA:tiltsNotSameLength";
    case RCABF_ERR_VS_NOT_SAME_LENGTH: return "bfVirtualSourceGeneric_RCA:virtualSourcesNotSameLength";
    case RCABF_ERR_THETA_OR_VS_INVALID: return "bfVirtualSourceGeneric_RCA:ThetaORVirtualSourceInvalid";
    case RCABF_ERR_FLAG_RECEIVE_X_INVALID: return "bfVirtualSourceGeneric_RCA:flagReceiveXInvalid";
    case RCABF_ERR_PARAM_NOT_STRUCT: return "bfVirtualSourceGeneric_RCA:ParamNotStruct";
    case RCABF_ERR_FS_MISSING: return "bfVirtualSourceGeneric_RCA:samplingFrequencyMissing";
    case RCABF_ERR_FS_INVALID: return "bfVirtualSourceGeneric_RCA:samplingFrequencyInvalid";
    case RCABF_ERR_FD_MISSING: return "bfVirtualSourceGeneric_RCA:demodulationFrequencyMissing";
    case RCABF_ERR_FD_INVALID: return "bfVirtualSourceGeneric_RCA:demodulationFrequencyInvalid";
    case RCABF_ERR_SPEED_OF_SOUND_INVALID: return "bfVirtualSourceGeneric_RCA:speedOfSoundInvalid";
    case RCABF_ERR_START_TIME_INVALID: return "bfVirtualSourceGeneric_RCA:startTimeInvalid";
    case RCABF_ERR_INVALID_ARGUMENT: return "rcabf:invalidArgument";
    case RCABF_ERR_SHAPE_MISMATCH: return "rcabf:shapeMismatch";
    case RCABF_ERR_UNSUPPORTED: return "rcabf:unsupported";
    case RCABF_ERR_WORKSPACE_TOO_SMALL: return "rcabf:workspaceTooSmall";
    case RCABF_ERR_OOM_ADMISSION: return "rcabf:oomAdmission";
    case RCABF_ERR_TIMEOUT: return "rcabf:timeout";
    case RCABF_ERR_CUDA: return "rcabf:cudaError";
    case RCABF_ERR_BOUNDS: return "rcabf:boundsCheck";
    case RCABF_ERR_BAD_HANDLE: return "rcabf:badHandle";
    case RCABF_ERR_CANCELLED: return "rcabf:cancelled";
    case RCABF_ERR_BUSY: return "rcabf:busy";
    case RCABF_ERR_PENDING: return "rcabf:pending";
    default: return "rcabf:unknown";
    }
}

int rcabf_abi_version(void) { return RCABF_ABI_VERSION; }

const char *rcabf_last_error(void) { return g_last_err; }

int rcabf_create_geometry(const rcabf_geometry_desc *desc, void *stream, rcabf_geometry **out)
{
    int s = build_geometry(desc, (cudaStream_t)stream, out);
    if (s == RCABF_OK) device_state((*out)->device);
    return s;
}

int rcabf_destroy_geometry(rcabf_geometry *g)
{
    if (!g) return RCABF_ERR_BAD_HANDLE;
    free_geometry(g);
    return RCABF_OK;
}

int rcabf_geometry_info(const rcabf_geometry *g, int64_t *n_pix, int64_t *n_tx, int64_t *n_ele)
{
    if (!g) return RCABF_ERR_BAD_HANDLE;
    if (n_pix) *n_pix = g->n_pix;
    if (n_tx) *n_tx = g->n_tx;
    if (n_ele) *n_ele = g->n_ele;
    return RCABF_OK;
}

int rcabf_geometry_sources(const rcabf_geometry *g, double *vs_x, double *vs_y, double *vs_z, double *min_dist)
{
    if (!g) return RCABF_ERR_BAD_HANDLE;
    for (int t = 0; t < g->n_tx; ++t) {
        if (vs_x) vs_x[t] = g->vs_x[t];
        if (vs_y) vs_y[t] = g->vs_y[t];
        if (vs_z) vs_z[t] = g->vs_z[t];
        if (min_dist) min_dist[t] = g->min_dist[t];
    }
    return RCABF_OK;
}

int rcabf_beamform_workspace_size(const rcabf_geometry *g, const rcabf_beamform_args *a, size_t *bytes)
{
    if (!bytes) return RCABF_ERR_INVALID_ARGUMENT;
    Plan p;
    int s = plan_beamform(const_cast<rcabf_geometry *>(g), a, p);
    if (s == RCABF_OK) *bytes = p.total;
    return s;
}

int rcabf_describe_plan(const rcabf_geometry *g, const rcabf_beamform_args *a, char *buf, size_t len)
{
    if (!buf || len == 0) return RCABF_ERR_INVALID_ARGUMENT;
    Plan p;
    int s = plan_beamform(const_cast<rcabf_geometry *>(g), a, p);
    if (s != RCABF_OK) return s;
    int occ = 0;   // resident CTAs per SM of the fused kernel (0: plain kernel)
    if (p.tc) {
        occ = 1;
    } else if (p.kernel == RCABF_KERNEL_FUSED) {
        s = resident_ctas(g, p, p.smem, device_state(g->device), occ);
        if (s != RCABF_OK) return s;
    }
    const char *kname = p.pc_all                         ? "per_channel_all_frames"
                        : p.kernel == RCABF_KERNEL_PLAIN ? "plain"
                        : p.tc == 2                     ? "fused_tensor_core"
                        : p.tc == 1                     ? "fused_tensor_core_fp16w"
                        : p.vb == 2                     ? "fused_voxel_blocked_tmem"
                        : p.vb                          ? "fused_voxel_blocked"
                                                        : "fused";
    // tensor-core plans: the MMA work of one call, counted on the host
    double mma_flops = 0.0;
    if (p.tc) {
        const int64_t chunks = const_cast<rcabf_geometry *>(g)->tc_chunks(p.ts, a->n_sample);
        const int nmat = p.tc == 2 ? 4 : 2;
        const int n16 = (2 * p.fb + 15) / 16 * 16;
        mma_flops = (double)chunks * p.n_fb * nmat * 2.0 * 128.0 * n16 * 16.0;   // nmat MMAs per chunk
    }
    snprintf(buf, len,
             "{\"kernel\": \"%s\", \"row_shift\": %d, \"frames_per_block\": %d, \"frame_blocks\": %d, "
             "\"tile\": [%d, %d, %d], \"voxels_per_thread\": %d, \"window_rows\": %d, \"smem_bytes\": %zu, "
             "\"workspace_bytes\": %zu, \"work_items\": %lld, \"storage\": %d, \"ctas_per_sm\": %d, "
             "\"mma_flops\": %.6e}",
             kname, p.d, p.fb, p.n_fb, p.ts.tu, p.vb ? p.ts.tv * VB_BLOCK : p.ts.tv, p.ts.tz, p.vb ? VB_BLOCK : 1,
             p.wmax, p.smem, p.total, (long long)p.n_items, p.store, occ, mma_flops);
    return RCABF_OK;
}

int rcabf_beamform(const rcabf_geometry *g, const rcabf_beamform_args *a, void *stream)
{
    if (!g) return RCABF_ERR_BAD_HANDLE;
    return beamform_one(const_cast<rcabf_geometry *>(g), a, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// Host-buffer beamforming: frames in chunks, copies overlapped with compute
// ---------------------------------------------------------------------------
namespace {

size_t iq_sample_bytes(int iq_dtype) { return iq_dtype == RCABF_IQ_C64 ? 8 : iq_dtype == RCABF_IQ_RF_F32 ? 8 : 4; }
size_t align256(size_t x) { return (x + 255) / 256 * 256; }

// Chunk length (whole frame blocks of the full call's plan, the last chunk
// the shortest) and the device buffers of two chunks in the workspace.
struct HostLayout {
    int64_t chunk = 0;
    size_t in_bytes = 0, out_bytes = 0, plan_bytes = 0, total = 0;
    bool have_tuned = false;   // the autotuner's choice for the whole call, used by every chunk
    TuneChoice tuned;
};

// Plan of one chunk: the whole call's tuned choice where one exists and fits.
int chunk_plan(rcabf_geometry *g, const rcabf_beamform_args *c, const HostLayout &h, Plan &p)
{
    if (h.have_tuned && plan_beamform(g, c, p, &h.tuned) == RCABF_OK) return RCABF_OK;
    return plan_beamform(g, c, p);
}

int host_layout(rcabf_geometry *g, const rcabf_beamform_args *a, int32_t frames_per_chunk, HostLayout &h)
{
    if (a->per_channel) return RCABF_ERR_UNSUPPORTED;   // [element][frame]... output: not frame-major
    if (frames_per_chunk < 0) return RCABF_ERR_INVALID_ARGUMENT;
    Plan p;
    int s = plan_beamform(g, a, p);
    if (s != RCABF_OK) return s;
    int64_t chunk = frames_per_chunk;
    if (chunk == 0) {
        // about four chunks of whole frame blocks: the first copy in and the
        // last copy out are the only transfers not hidden under compute
        const int64_t fb = p.kernel == RCABF_KERNEL_FUSED ? p.fb : 1;
        const int64_t n_fb = (a->n_frame + fb - 1) / fb;
        chunk = fb * ((n_fb + 3) / 4);
    }
    h.chunk = std::min<int64_t>(chunk, a->n_frame);
    {
        std::lock_guard<std::mutex> lk(g->mu);
        auto it = g->tuned.find({a->n_frame, (int64_t)a->storage});
        if (it != g->tuned.end() && p.kernel == RCABF_KERNEL_FUSED && it->second.fb == p.fb && it->second.vb == p.vb) {
            h.have_tuned = true;
            h.tuned = it->second;
        }
    }
    if (p.tc && !h.have_tuned) {   // every chunk on the tensor-core kernel (its frame block its own)
        h.have_tuned = true;
        h.tuned = TuneChoice{};
        h.tuned.tc = p.tc;
        h.tuned.ts = p.ts;
    }
    const int64_t n_t = a->compound ? 1 : a->n_tx;
    h.in_bytes = align256((size_t)h.chunk * a->n_tx * a->n_ch * a->n_sample * iq_sample_bytes(a->iq_dtype));
    h.out_bytes = align256((size_t)h.chunk * n_t * g->n_pix * 8);
    rcabf_beamform_args c = *a;
    c.n_frame = h.chunk;
    Plan pc;
    if ((s = chunk_plan(g, &c, h, pc)) != RCABF_OK) return s;
    h.plan_bytes = align256(pc.total);
    h.total = 2 * h.in_bytes + 2 * h.out_bytes + h.plan_bytes;
    return RCABF_OK;
}

}  // namespace

int rcabf_beamform_host_workspace_size(const rcabf_geometry *g, const rcabf_beamform_args *a,
                                       int32_t frames_per_chunk, size_t *bytes)
{
    if (!g) return RCABF_ERR_BAD_HANDLE;
    if (!a || !bytes) return RCABF_ERR_INVALID_ARGUMENT;
    HostLayout h;
    const int s = host_layout(const_cast<rcabf_geometry *>(g), a, frames_per_chunk, h);
    if (s == RCABF_OK) *bytes = h.total;
    return s;
}

int rcabf_beamform_host(const rcabf_geometry *g0, const rcabf_beamform_args *a, int32_t frames_per_chunk,
                        void *stream)
{
    if (!g0) return RCABF_ERR_BAD_HANDLE;
    if (!a || !a->iq || !a->out) return RCABF_ERR_INVALID_ARGUMENT;
    rcabf_geometry *g = const_cast<rcabf_geometry *>(g0);
    HostLayout h;
    int s = host_layout(g, a, frames_per_chunk, h);
    if (s != RCABF_OK) return s;
    if (a->workspace_bytes < h.total || !a->workspace) return RCABF_ERR_WORKSPACE_TOO_SMALL;
    if (((uintptr_t)a->workspace) % 256) return RCABF_ERR_INVALID_ARGUMENT;
    char *ws = static_cast<char *>(a->workspace);
    char *dev_in[2] = {ws, ws + h.in_bytes};
    char *dev_out[2] = {ws + 2 * h.in_bytes, ws + 2 * h.in_bytes + h.out_bytes};
    char *plan_ws = ws + 2 * h.in_bytes + 2 * h.out_bytes;
    const cudaStream_t st = (cudaStream_t)stream;
    const size_t in_frame = (size_t)a->n_tx * a->n_ch * a->n_sample * iq_sample_bytes(a->iq_dtype);
    const size_t out_frame = (size_t)(a->compound ? 1 : a->n_tx) * g->n_pix * 8;

    // copy-in and copy-out streams; events order the three per buffer slot
    cudaStream_t cin = nullptr, cout = nullptr;
    cudaEvent_t ev[7] = {};   // start, in_ready[2], done[2], out_done[2]
    auto cleanup = [&]() {
        for (cudaEvent_t e : ev)
            if (e) cudaEventDestroy(e);   // released once pending work that uses it completes
        if (cin) cudaStreamDestroy(cin);
        if (cout) cudaStreamDestroy(cout);
    };
    cudaError_t ce = cudaStreamCreateWithFlags(&cin, cudaStreamNonBlocking);
    if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&cout, cudaStreamNonBlocking);
    for (int i = 0; i < 7 && ce == cudaSuccess; ++i) ce = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming);
    if (ce != cudaSuccess) { cleanup(); return cuda_fail(ce, "host pipeline streams"); }
    cudaEvent_t start = ev[0], *in_ready = ev + 1, *done = ev + 3, *out_done = ev + 5;
    // the copies follow the caller's earlier work on `stream`
    ce = cudaEventRecord(start, st);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(cin, start, 0);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(cout, start, 0);

    const char *host_in = static_cast<const char *>(a->iq);
    char *host_out = static_cast<char *>(a->out);
    for (int64_t f0 = 0, c = 0; f0 < a->n_frame && ce == cudaSuccess && s == RCABF_OK; f0 += h.chunk, ++c) {
        const int b = (int)(c % 2);
        const int64_t nf = std::min<int64_t>(h.chunk, a->n_frame - f0);
        // in: slot b is free once chunk c - 2 is computed (and copied out,
        // when the output chunk is loaded for accumulation)
        if (c >= 2) ce = cudaStreamWaitEvent(cin, done[b], 0);
        if (ce == cudaSuccess && c >= 2 && a->accumulate) ce = cudaStreamWaitEvent(cin, out_done[b], 0);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(dev_in[b], host_in + f0 * in_frame, nf * in_frame, cudaMemcpyHostToDevice, cin);
        if (ce == cudaSuccess && a->accumulate)
            ce = cudaMemcpyAsync(dev_out[b], host_out + f0 * out_frame, nf * out_frame, cudaMemcpyHostToDevice, cin);
        if (ce == cudaSuccess) ce = cudaEventRecord(in_ready[b], cin);
        // compute on the caller's stream, into slot b once its last copy-out ended
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st, in_ready[b], 0);
        if (ce == cudaSuccess && c >= 2 && !a->accumulate) ce = cudaStreamWaitEvent(st, out_done[b], 0);
        if (ce != cudaSuccess) break;
        rcabf_beamform_args ca = *a;
        ca.iq = dev_in[b];
        ca.out = dev_out[b];
        ca.n_frame = nf;
        ca.mask = c == 0 ? a->mask : nullptr;   // the mask does not depend on frames: once
        ca.workspace = plan_ws;
        ca.workspace_bytes = h.plan_bytes;
        ca.stage_events = nullptr;
        Plan pc;
        s = chunk_plan(g, &ca, h, pc);
        if (s == RCABF_OK) s = beamform_planned(g, &ca, pc, st);
        if (s != RCABF_OK) break;
        ce = cudaEventRecord(done[b], st);
        // out
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(cout, done[b], 0);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(host_out + f0 * out_frame, dev_out[b], nf * out_frame, cudaMemcpyDeviceToHost, cout);
        if (ce == cudaSuccess) ce = cudaEventRecord(out_done[b], cout);
    }
    // the caller's stream completes after the last copies out
    if (ce == cudaSuccess) ce = cudaEventRecord(out_done[0], cout);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st, out_done[0], 0);
    if (ce != cudaSuccess || s != RCABF_OK) {
        // no copy may still touch the caller's host buffers after an error return
        cudaStreamSynchronize(cin);
        cudaStreamSynchronize(cout);
    }
    cleanup();
    if (ce != cudaSuccess) return cuda_fail(ce, "host pipeline");
    return s;
}

int rcabf_beamform_noalloc(const rcabf_geometry *g, const rcabf_beamform_args *a, void *stream)
{
    if (!g) return RCABF_ERR_BAD_HANDLE;
    return beamform_noalloc(const_cast<rcabf_geometry *>(g), a, (cudaStream_t)stream);
}

int rcabf_beamform_batch(int n, const rcabf_geometry *const *gs, const rcabf_beamform_args *as, void *stream)
{
    if (n < 1 || n > MAX_JOBS || !gs || !as) return RCABF_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    rcabf_geometry *g0 = const_cast<rcabf_geometry *>(gs[0]);
    if (!g0) return RCABF_ERR_BAD_HANDLE;
    FusedParams prm{};
    Plan p0;
    int64_t items = 0;
    int wmax = 0;
    for (int i = 0; i < n; ++i) {
        rcabf_geometry *g = const_cast<rcabf_geometry *>(gs[i]);
        if (!g) return RCABF_ERR_BAD_HANDLE;
        if (as[i].frames_per_block <= 0 || as[i].frames_per_block != as[0].frames_per_block)
            return RCABF_ERR_INVALID_ARGUMENT;
        if (as[i].kernel == RCABF_KERNEL_PLAIN) return RCABF_ERR_INVALID_ARGUMENT;
        if (g->mode != g0->mode || g->kind != g0->kind || g->device != g0->device ||
            as[i].storage != as[0].storage)
            return RCABF_ERR_UNSUPPORTED;
        Plan p;
        int s = plan_beamform(g, &as[i], p);
        if (s != RCABF_OK) return s;
        if ((s = check_ptrs(&as[i], p)) != RCABF_OK) return s;
        if (i == 0) p0 = p;
        // one launch = one kernel variant: every job fused, same frame block
        if (p.kernel != RCABF_KERNEL_FUSED || p.fb != p0.fb || p.vb != p0.vb || p.d != p0.d)
            return RCABF_ERR_UNSUPPORTED;
        wmax = std::max(wmax, p.wmax);
        if ((s = stage_job(g, &as[i], p, prm.jobs[i], st)) != RCABF_OK) return s;
        prm.jobs[i].item_begin = items;
        items += p.n_items;
    }
    prm.n_jobs = n;
    prm.wmax = wmax;
    prm.row_words = p0.row_words;
    prm.n_items = items;
    int s = launch_fused_jobs(g0, prm, p0, st);
    if (s != RCABF_OK) return s;
    for (int i = 0; i < n; ++i) {
        if (!as[i].mask) continue;
        const cudaError_t me = launch_mask(gs[i]->dev(), as[i].mask, as[i].compound ? 1 : 0, as[i].accumulate ? 1 : 0, st);
        if (me != cudaSuccess) return cuda_fail(me, "mask kernel launch");
        g_launches += 1;
    }
    return RCABF_OK;
}

int rcabf_autotune(const rcabf_geometry *gc, const rcabf_beamform_args *a, void *stream, int iters,
                   rcabf_tune_result *res)
{
    if (!gc) return RCABF_ERR_BAD_HANDLE;
    if (!a || !res || res->struct_size != (int32_t)sizeof(rcabf_tune_result) || iters < 1 || iters > 100)
        return RCABF_ERR_INVALID_ARGUMENT;
    if (a->kernel == RCABF_KERNEL_PLAIN) return RCABF_ERR_UNSUPPORTED;
    rcabf_geometry *g = const_cast<rcabf_geometry *>(gc);
    cudaStream_t st = (cudaStream_t)stream;
    // the candidates overwrite out; nothing accumulates, no mask, no stage events
    rcabf_beamform_args b = *a;
    b.accumulate = 0;
    b.mask = nullptr;
    b.stage_events = nullptr;
    b.frames_per_block = 0;
    b.workspace = nullptr;
    b.workspace_bytes = 0;
    const std::array<int64_t, 2> key{a->n_frame, (int64_t)a->storage};
    {
        std::lock_guard<std::mutex> lk(g->mu);
        g->tuned.erase(key);   // measure from the planner's own choice
    }
    Plan p0;
    int s = plan_beamform(g, &b, p0);
    if (s != RCABF_OK) return s;
    if (p0.kernel != RCABF_KERNEL_FUSED) return RCABF_ERR_UNSUPPORTED;

    void *ws = nullptr;
    size_t ws_bytes = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return cuda_fail(cudaGetLastError(), "autotune events");
    int tried = 0;
    auto time_plan = [&](const Plan &p, double &ms) -> int {
        if (p.total > ws_bytes) {
            if (ws) cudaFree(ws);
            ws = nullptr;
            ws_bytes = 0;
            const cudaError_t me = cudaMalloc(&ws, p.total);
            if (me != cudaSuccess) { cudaGetLastError(); return RCABF_ERR_WORKSPACE_TOO_SMALL; }
            ws_bytes = p.total;
        }
        b.workspace = ws;
        b.workspace_bytes = ws_bytes;
        int r = beamform_planned(g, &b, p, st);   // first run: kernel attributes, caches
        if (r != RCABF_OK) return r;
        cudaEventRecord(e0, st);
        for (int i = 0; i < iters && r == RCABF_OK; ++i) r = beamform_planned(g, &b, p, st);
        cudaEventRecord(e1, st);
        if (r != RCABF_OK) return r;
        const cudaError_t se = cudaEventSynchronize(e1);
        if (se != cudaSuccess) return cuda_fail(se, "autotune");
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms = t / iters;
        ++tried;
        return RCABF_OK;
    };

    double default_ms = 0.0;
    s = time_plan(p0, default_ms);
    TuneChoice best{p0.vb, p0.fb, p0.ts, p0.tc};
    double best_ms = default_ms;
    auto consider = [&](const TuneChoice &c) {
        Plan p;
        if (plan_beamform(g, &b, p, &c) != RCABF_OK) return;   // does not fit
        double ms = 0.0;
        if (time_plan(p, ms) != RCABF_OK) { cudaGetLastError(); return; }
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
            best.fb = p.fb;   // the frame block the choice planned (the tensor-core kernel picks its own)
        }
    };
    if (s == RCABF_OK) {
        if (p0.vb) {
            // tile shapes (lanes along u, voxel blocks along v, depth) at the
            // planner's frame block, then frame blocks at the best tile
            const TileShape tiles[] = {{4, 2, 16}, {2, 4, 16}, {4, 4, 8}, {8, 2, 8}, {2, 2, 32}, {8, 1, 16},
                                       {4, 1, 32}, {1, 4, 32}};
            for (const TileShape &t : tiles) {
                if (t.tu == p0.ts.tu && t.tv == p0.ts.tv && t.tz == p0.ts.tz) continue;
                consider(TuneChoice{p0.vb, p0.fb, t});
            }
            const TileShape bt = best.ts;
            for (int fb : {2, 4, 8, 16}) {
                if (fb == p0.fb || fb > 2 * a->n_frame) continue;
                consider(TuneChoice{p0.vb, fb, bt});
            }
            // the other accumulator store (registers / tensor memory) at every
            // frame block
            for (int fb : {2, 4, 8, 16}) {
                if (fb > 2 * a->n_frame) continue;
                consider(TuneChoice{p0.vb == 2 ? 1 : 2, fb, bt});
            }
        }
        // the tensor-core kernel (hi + remainder weights) where it applies
        if (!p0.tc) {
            TuneChoice tcc;
            tcc.tc = 2;
            consider(tcc);
        }
        // the one-voxel-per-thread kernel at its own frame blocks
        rcabf_beamform_args nb = b;
        nb.kernel = RCABF_KERNEL_FUSED_NOBLOCK;
        Plan pn;
        if (plan_beamform(g, &nb, pn) == RCABF_OK && pn.kernel == RCABF_KERNEL_FUSED) {
            for (int fb : {pn.fb, 40, 16}) {
                if (!fb_supported(g->mode, fb) || (fb != pn.fb && fb > 2 * a->n_frame)) continue;
                if (!p0.vb && fb == p0.fb) continue;   // the default itself
                consider(TuneChoice{0, fb, pn.ts});
            }
        }
    }
    if (ws) cudaFree(ws);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != RCABF_OK) return s;
    {
        std::lock_guard<std::mutex> lk(g->mu);
        g->tuned[key] = best;
    }
    Plan pb;
    plan_beamform(g, &b, pb);
    res->voxel_blocked = pb.vb;
    res->frames_per_block = pb.fb;
    res->tile_u = pb.ts.tu;
    res->tile_v = pb.vb ? pb.ts.tv * VB_BLOCK : pb.ts.tv;
    res->tile_z = pb.ts.tz;
    res->window_rows = pb.wmax;
    res->candidates = tried;
    res->best_ms = best_ms;
    res->default_ms = default_ms;
    res->tensor_core = pb.tc ? 1 : 0;
    return RCABF_OK;
}

int rcabf_take_error_count(int64_t *count)
{
    if (!count) return RCABF_ERR_INVALID_ARGUMENT;
    int dev = 0;
    cudaGetDevice(&dev);
    DeviceState *ds = device_state(dev);
    unsigned long long h = 0;
    if (!ds->err) return RCABF_ERR_CUDA;
    if (cudaMemcpy(&h, ds->err, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return RCABF_ERR_CUDA;
    if (cudaMemset(ds->err, 0, sizeof(h)) != cudaSuccess) return RCABF_ERR_CUDA;
    NoallocRegion r;   // plus the static counter of rcabf_beamform_noalloc, once set up
    if (noalloc_setup(dev, r, false) == RCABF_OK) {
        unsigned long long h2 = 0;
        if (cudaMemcpy(&h2, r.err, sizeof(h2), cudaMemcpyDeviceToHost) != cudaSuccess) return RCABF_ERR_CUDA;
        if (cudaMemset(r.err, 0, sizeof(h2)) != cudaSuccess) return RCABF_ERR_CUDA;
        h += h2;
    }
    *count = (int64_t)h;
    return RCABF_OK;
}

int rcabf_take_launch_count(int64_t *count)
{
    if (!count) return RCABF_ERR_INVALID_ARGUMENT;
    *count = g_launches.exchange(0);
    return RCABF_OK;
}

int rcabf_measure_fp32_peak(double *tflops, void *stream)
{
    if (!tflops) return RCABF_ERR_INVALID_ARGUMENT;
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    cudaGetDevice(&dev);
    DeviceState *ds = device_state(dev);
    float *out = nullptr;
    if (cudaMalloc(&out, 256 * sizeof(float)) != cudaSuccess) return RCABF_ERR_CUDA;
    const int blocks = ds->n_sm * 8, iters = 4096;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch_fma_probe(out, blocks, 64, st);  // warm-up
    cudaEventRecord(e0, st);
    launch_fma_probe(out, blocks, iters, st);
    cudaEventRecord(e1, st);
    cudaError_t ce = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (ce != cudaSuccess || ms <= 0.f) return RCABF_ERR_CUDA;
    const double flops = 2.0 * 8 * 16 * (double)iters * 256.0 * blocks;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return RCABF_OK;
}

}  // extern "C"
