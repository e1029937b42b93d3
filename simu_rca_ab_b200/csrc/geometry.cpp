// Geometry construction: validation of the acquisition description, the
// reference wrapper's host preprocessing (element centring, apertures,
// virtual sources, minimum source-to-array distance), and the separable
// delay tables.
//
// RCA separability: with receive on the X (column) elements and transmit on
// the Y (row) elements (flagReceiveX, RCA.cu:256-262, 284-291), the transmit
// delay depends on (y, z) only and the receive delay on (x, z) only; with
// receive on Y the roles swap.  The tables are therefore indexed by
//   rx key (u, z): u = the receive axis coordinate, one row per element,
//   tx key (v, z): v = the transmit steering axis, one row per transmit,
// instead of per voxel.
#include "geometry.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>

#include "launchers.h"

namespace rcabf {

static bool all_finite(const double *p, int64_t n)
{
    for (int64_t i = 0; i < n; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

// Angle between AB and AC (RCA.cu:85-98, in double).
static double angle_ab_ac(double ax, double ay, double bx, double by, double cx, double cy)
{
    const double abx = bx - ax, aby = by - ay, acx = cx - ax, acy = cy - ay;
    const double den = std::sqrt((abx * abx + aby * aby) * (acx * acx + acy * acy));
    double cs = (abx * acx + aby * acy) / den;
    cs = std::max(-1.0, std::min(1.0, cs));
    return std::acos(cs);
}

// Transmit cone along one lateral axis (RCA.cu:193-214): the point (p, z)
// lies inside the cone from the source (vl, vz) through the edges (+-h, -az).
static bool cone_half(double vl, double vz, double h, double az, double p, double z)
{
    const double cone = angle_ab_ac(vl, vz, -h, -az, h, -az);
    return angle_ab_ac(vl, vz, -h, -az, p, z) <= cone && angle_ab_ac(vl, vz, h, -az, p, z) <= cone;
}

static inline void unit_phasor(double cycles, float &c, float &s)
{
    const double r = cycles - std::nearbyint(cycles);
    c = (float)std::cos(2.0 * M_PI * r);
    s = (float)std::sin(2.0 * M_PI * r);
}

// Polyphase weight table of a windowed-sinc kernel, sinc(x) sinc(x / W) at
// x_j = d + LO - j (RCA.cu:331-336 for W = 2, 6 taps; Lanczos-a for W = a,
// zero for |x| >= a): WT_Q rows of 16 floats, the weights at d = q / WT_Q
// then their increments to d = (q + 1) / WT_Q, evaluated in FP64.
static std::vector<float> weight_table(int kind)
{
    const int Q = 256, ROW = 16;
    const int taps = kind_taps(kind), lo = kind_lo(kind);
    const double W = kind == K_REF6 ? 2.0 : kind == K_LANCZOS2 ? 2.0 : kind == K_LANCZOS3 ? 3.0 : 4.0;
    const bool lanczos = kind != K_REF6;
    auto sinc = [](double x) { return x == 0.0 ? 1.0 : std::sin(M_PI * x) / (M_PI * x); };
    auto w = [&](double d, int j) {
        const double x = d + lo - j;
        if (lanczos && std::fabs(x) >= W) return 0.0;
        return sinc(x) * sinc(x / W);
    };
    std::vector<float> t((size_t)Q * ROW, 0.f);
    for (int q = 0; q < Q; ++q)
        for (int j = 0; j < taps; ++j) {
            const double a = w((double)q / Q, j), b = w((double)(q + 1) / Q, j);
            t[(size_t)q * ROW + j] = (float)a;
            t[(size_t)q * ROW + 8 + j] = (float)(b - a);
        }
    return t;
}

template <typename T>
static cudaError_t upload(T **dst, const std::vector<T> &src, cudaStream_t st)
{
    if (src.empty()) { *dst = nullptr; return cudaSuccess; }
    cudaError_t e = cudaMalloc((void **)dst, src.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st);
}

void free_geometry(rcabf_geometry *g)
{
    if (!g) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    cudaFree(g->rx_tab);
    cudaFree(g->tx_tab);
    cudaFree(g->cone_u);
    cudaFree(g->apod_sum);
    cudaFree(g->ab);
    cudaFree(g->ab_ph);
    cudaFree(g->wtab);
    cudaSetDevice(prev);
    delete g;
}

int build_geometry(const rcabf_geometry_desc *d, cudaStream_t st, rcabf_geometry **out)
{
    if (!d || !out) return RCABF_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (d->struct_size != (int32_t)sizeof(rcabf_geometry_desc)) return RCABF_ERR_INVALID_ARGUMENT;

    // ---- validation (reference error identifiers where one applies) ----
    if (d->n_ele < 1 || !d->pos_ele_x || !d->pos_ele_y || !d->pos_ele_z) return RCABF_ERR_POS_ELE_INVALID;
    if (!all_finite(d->pos_ele_x, d->n_ele) || !all_finite(d->pos_ele_y, d->n_ele) ||
        !all_finite(d->pos_ele_z, d->n_ele))
        return RCABF_ERR_POS_ELE_INVALID;
    if (d->n_ele > (1 << 20)) return RCABF_ERR_UNSUPPORTED;
    if (d->grid_kind == RCABF_GRID_RECTILINEAR) {
        if (d->n_z < 1 || d->n_x < 1 || d->n_y < 1 || !d->grid_x || !d->grid_y || !d->grid_z)
            return RCABF_ERR_GRID_INVALID;
        if (!all_finite(d->grid_x, d->n_x) || !all_finite(d->grid_y, d->n_y) || !all_finite(d->grid_z, d->n_z))
            return RCABF_ERR_GRID_INVALID;
    } else if (d->grid_kind == RCABF_GRID_POINTS) {
        if (d->n_z < 1 || d->n_x != 1 || d->n_y != 1 || !d->grid_x || !d->grid_y || !d->grid_z)
            return RCABF_ERR_GRID_INVALID;
        if (!all_finite(d->grid_x, d->n_z) || !all_finite(d->grid_y, d->n_z) || !all_finite(d->grid_z, d->n_z))
            return RCABF_ERR_GRID_INVALID;
    } else {
        return RCABF_ERR_GRID_INVALID;
    }
    if (d->n_tx < 1) return RCABF_ERR_THETA_OR_VS_REQUIRED;
    if (d->n_tx > 65535) return RCABF_ERR_UNSUPPORTED;
    if (d->use_theta) {
        if (!d->theta_x || !d->theta_y) return RCABF_ERR_THETA_OR_VS_INVALID;
        if (!all_finite(d->theta_x, d->n_tx) || !all_finite(d->theta_y, d->n_tx)) return RCABF_ERR_THETA_OR_VS_INVALID;
    } else {
        if (!d->vs_x || !d->vs_y || !d->vs_z) return RCABF_ERR_THETA_OR_VS_INVALID;
        if (!all_finite(d->vs_x, d->n_tx) || !all_finite(d->vs_y, d->n_tx) || !all_finite(d->vs_z, d->n_tx))
            return RCABF_ERR_THETA_OR_VS_INVALID;
    }
    if (!std::isfinite(d->fs) || !(d->fs > 0)) return RCABF_ERR_FS_INVALID;
    if (!std::isfinite(d->fd)) return RCABF_ERR_FD_INVALID;
    if (!std::isfinite(d->c) || !(d->c > 0)) return RCABF_ERR_SPEED_OF_SOUND_INVALID;
    if (!std::isfinite(d->t0)) return RCABF_ERR_START_TIME_INVALID;
    // The reference reports an invalid f-number with the start-time identifier (RCA.m:449-454).
    if (std::isnan(d->fnumber) || std::isinf(d->fnumber)) return RCABF_ERR_START_TIME_INVALID;
    if (std::isnan(d->aperture_x) == false && !std::isfinite(d->aperture_x)) return RCABF_ERR_APERTURE_X_INVALID;
    if (std::isnan(d->aperture_y) == false && !std::isfinite(d->aperture_y)) return RCABF_ERR_APERTURE_Y_INVALID;
    if (std::isnan(d->aperture_z) == false && !std::isfinite(d->aperture_z)) return RCABF_ERR_APERTURE_Z_INVALID;
    int kind;
    switch (d->interp) {
    case RCABF_INTERP_QUAD3: kind = K_QUAD3; break;
    case RCABF_INTERP_REF6: kind = K_REF6; break;
    case RCABF_INTERP_LANCZOS:
        if (d->lanczos_a == 2) kind = K_LANCZOS2;
        else if (d->lanczos_a == 3) kind = K_LANCZOS3;
        else if (d->lanczos_a == 4) kind = K_LANCZOS4;
        else return RCABF_ERR_INTERPOLATION_INVALID;
        break;
    default: return RCABF_ERR_INTERPOLATION_INVALID;
    }
    if (d->table_mode != RCABF_TABLES_EXACT && d->table_mode != RCABF_TABLES_REF_COMPAT)
        return RCABF_ERR_INVALID_ARGUMENT;
    const int mode = d->table_mode == RCABF_TABLES_REF_COMPAT ? MODE_REF : MODE_EXACT;
    if (mode == MODE_REF && kind != K_QUAD3 && kind != K_REF6) return RCABF_ERR_UNSUPPORTED;
    if (d->ab_law) {
        const int64_t n_ab = d->ab_per_tx ? d->n_tx * d->n_ele : d->n_ele;
        if (!all_finite(d->ab_law, n_ab)) return RCABF_ERR_INVALID_ARGUMENT;
    }

    std::unique_ptr<rcabf_geometry> g(new rcabf_geometry());
    cudaGetDevice(&g->device);
    g->mode = mode;
    g->interp = d->interp;
    g->lanczos_a = d->lanczos_a;
    g->kind = kind;
    g->receive_x = d->receive_x ? 1 : 0;
    g->mask_transmit = d->mask_transmit ? 1 : 0;
    g->grid_kind = d->grid_kind;
    g->fs = d->fs; g->fd = d->fd; g->c = d->c; g->t0 = d->t0; g->fnumber = d->fnumber;
    const int64_t ne = d->n_ele, nt = d->n_tx;
    g->n_ele = (int)ne;
    g->n_tx = (int)nt;

    // ---- elements centred on their mean (RCA.m:500-502) ----
    auto centred = [&](const double *p) {
        double m = 0;
        for (int64_t i = 0; i < ne; ++i) m += p[i];
        m /= (double)ne;
        std::vector<double> v(ne);
        for (int64_t i = 0; i < ne; ++i) v[i] = p[i] - m;
        return v;
    };
    const std::vector<double> ex = centred(d->pos_ele_x), ey = centred(d->pos_ele_y), ez = centred(d->pos_ele_z);
    auto span = [&](const std::vector<double> &v) {
        return *std::max_element(v.begin(), v.end()) - *std::min_element(v.begin(), v.end());
    };
    // ---- apertures: given, else span of the centred positions (RCA.m:505-521) ----
    g->ap_x = std::isnan(d->aperture_x) ? span(ex) : d->aperture_x;
    g->ap_y = std::isnan(d->aperture_y) ? span(ey) : d->aperture_y;
    g->ap_z = std::isnan(d->aperture_z) ? span(ez) : d->aperture_z;

    // ---- virtual sources (RCA.m:527-547) ----
    g->vs_x.resize(nt); g->vs_y.resize(nt); g->vs_z.resize(nt); g->min_dist.resize(nt);
    for (int64_t s = 0; s < nt; ++s) {
        if (d->use_theta) {
            const double r = 10.0, tx = std::tan(d->theta_x[s]), ty = std::tan(d->theta_y[s]);
            g->vs_z[s] = -r / std::sqrt(1.0 + tx * tx + ty * ty);
            g->vs_x[s] = g->vs_z[s] * tx;
            g->vs_y[s] = g->vs_z[s] * ty;
        } else {
            g->vs_x[s] = d->vs_x[s]; g->vs_y[s] = d->vs_y[s]; g->vs_z[s] = d->vs_z[s];
        }
    }
    // ---- minimum distance from each source to the array (RCA.m:551-558).
    // The reference pairs the element Y positions with the source X and the
    // element X positions with the source Y; kept as is (it equals the true
    // distance to the transmitting row of a square RCA probe). ----
    for (int64_t s = 0; s < nt; ++s) {
        double m = std::numeric_limits<double>::infinity();
        for (int64_t k = 0; k < ne; ++k) {
            const double a = ey[k] - g->vs_x[s], b = ex[k] - g->vs_y[s], c = ez[k] - g->vs_z[s];
            m = std::min(m, std::sqrt(a * a + b * b + c * c));
        }
        g->min_dist[s] = m;
    }

    // ---- tile space and table keys ----
    const bool rxx = g->receive_x != 0;
    std::vector<double> key_u, key_v, key_z;  // rx keys: (u, z); tx keys: (v, z)
    int64_t n_rxkey, n_txkey;
    if (d->grid_kind == RCABF_GRID_RECTILINEAR) {
        g->n_z = d->n_z;
        g->n_u = rxx ? d->n_x : d->n_y;
        g->n_v = rxx ? d->n_y : d->n_x;
        g->s_z = d->stride_z;
        g->s_u = rxx ? d->stride_x : d->stride_y;
        g->s_v = rxx ? d->stride_y : d->stride_x;
        g->n_pix = d->n_z * d->n_x * d->n_y;
        const double *gu = rxx ? d->grid_x : d->grid_y;
        const double *gv = rxx ? d->grid_y : d->grid_x;
        key_u.assign(gu, gu + g->n_u);
        key_v.assign(gv, gv + g->n_v);
        key_z.assign(d->grid_z, d->grid_z + g->n_z);
        n_rxkey = g->n_u * g->n_z;
        n_txkey = g->n_v * g->n_z;
    } else {
        g->n_z = d->n_z; g->n_u = 1; g->n_v = 1;
        g->s_z = 1; g->s_u = 0; g->s_v = 0;
        g->n_pix = d->n_z;
        const double *gu = rxx ? d->grid_x : d->grid_y;
        const double *gv = rxx ? d->grid_y : d->grid_x;
        key_u.assign(gu, gu + d->n_z);
        key_v.assign(gv, gv + d->n_z);
        key_z.assign(d->grid_z, d->grid_z + d->n_z);
        n_rxkey = n_txkey = d->n_z;
    }
    // output strides must address [0, n_pix)
    if (d->grid_kind == RCABF_GRID_RECTILINEAR) {
        const int64_t last = (g->n_z - 1) * g->s_z + (g->n_u - 1) * g->s_u + (g->n_v - 1) * g->s_v;
        if (g->s_z < 0 || g->s_u < 0 || g->s_v < 0 || last >= g->n_pix) return RCABF_ERR_GRID_INVALID;
    }
    auto rk_u = [&](int64_t k) { return d->grid_kind == RCABF_GRID_RECTILINEAR ? key_u[k / g->n_z] : key_u[k]; };
    auto tk_v = [&](int64_t k) { return d->grid_kind == RCABF_GRID_RECTILINEAR ? key_v[k / g->n_z] : key_v[k]; };
    auto k_z = [&](int64_t k) { return d->grid_kind == RCABF_GRID_RECTILINEAR ? key_z[k % g->n_z] : key_z[k]; };

    const std::vector<double> &ele_u = rxx ? ex : ey;
    const std::vector<double> &vs_u = rxx ? g->vs_x : g->vs_y;
    const std::vector<double> &vs_v = rxx ? g->vs_y : g->vs_x;
    const double half_u = 0.5 * (rxx ? g->ap_x : g->ap_y), half_v = 0.5 * (rxx ? g->ap_y : g->ap_x);

    cudaError_t ce = cudaSuccess;
    g->rx_delay.assign((size_t)(ne * n_rxkey), 0.f);
    g->tx_delay.assign((size_t)(nt * n_txkey), 0.f);

    if (mode == MODE_EXACT) {
        // ---- FP64 tables ----
        const double F = g->fnumber, c = g->c, fs = g->fs, fd = g->fd;
        std::vector<float4> rx_tab((size_t)(ne * n_rxkey));
        std::vector<double> apod_sum_d((size_t)n_rxkey, 0.0);
        for (int64_t r = 0; r < ne; ++r)
            for (int64_t k = 0; k < n_rxkey; ++k) {
                const double u = rk_u(k), z = k_z(k);
                const double ap = std::fabs(u - ele_u[r]);
                const double apf = z / F;
                const bool valid = ap < apf;
                const double apod = valid ? 0.5 * (1.0 + std::cos(M_PI * ap / apf)) : 0.0;
                const double dz = z - ez[r];
                const double irx = std::sqrt(ap * ap + dz * dz) / c * fs;
                float pc, ps;
                unit_phasor(fd / fs * irx, pc, ps);
                float4 e;
                e.x = valid ? (float)irx : -1e30f;
                e.y = (float)(apod * pc);
                e.z = (float)(apod * ps);
                e.w = (float)apod;
                if (valid && !(e.w > 0.0f)) e.x = -1e30f;  // apodisation below float range
                rx_tab[r * n_rxkey + k] = e;
                apod_sum_d[k] += apod;
                g->rx_delay[r * n_rxkey + k] = (e.w > 0.0f) ? (float)irx : NAN;
            }
        std::vector<float4> tx_tab((size_t)(nt * n_txkey));
        for (int64_t t = 0; t < nt; ++t)
            for (int64_t k = 0; k < n_txkey; ++k) {
                const double v = tk_v(k), z = k_z(k);
                const double dv = v - vs_v[t], dz = z - g->vs_z[t];
                const double dtx = (std::sqrt(dv * dv + dz * dz) - g->min_dist[t]) / c;
                const double itx = (dtx + g->t0) * fs;
                float pc, ps;
                unit_phasor(fd / fs * itx - 2.0 * fd * z / c, pc, ps);
                const bool cone = !g->mask_transmit || cone_half(vs_v[t], g->vs_z[t], half_v, g->ap_z, v, z);
                tx_tab[t * n_txkey + k] = make_float4((float)itx, pc, ps, cone ? 1.f : 0.f);
                g->tx_delay[t * n_txkey + k] = (float)itx;
            }
        std::vector<float> apod_sum(apod_sum_d.begin(), apod_sum_d.end());
        if ((ce = upload(&g->rx_tab, rx_tab, st)) != cudaSuccess) goto cuda_fail;
        if ((ce = upload(&g->tx_tab, tx_tab, st)) != cudaSuccess) goto cuda_fail;
        if ((ce = upload(&g->apod_sum, apod_sum, st)) != cudaSuccess) goto cuda_fail;
        if (g->mask_transmit) {
            std::vector<uint8_t> cu((size_t)(nt * n_rxkey));
            for (int64_t t = 0; t < nt; ++t)
                for (int64_t k = 0; k < n_rxkey; ++k)
                    cu[t * n_rxkey + k] = cone_half(vs_u[t], g->vs_z[t], half_u, g->ap_z, rk_u(k), k_z(k)) ? 1 : 0;
            if ((ce = upload(&g->cone_u, cu, st)) != cudaSuccess) goto cuda_fail;
        }
        if (d->ab_law) {
            const int64_t n_ab = d->ab_per_tx ? nt * ne : ne;
            std::vector<float> ab((size_t)n_ab);
            std::vector<float2> abp((size_t)n_ab);
            for (int64_t i = 0; i < n_ab; ++i) {
                ab[i] = (float)(d->ab_law[i] * fs);
                float pc, ps;
                unit_phasor(fd * d->ab_law[i], pc, ps);
                abp[i] = make_float2(pc, ps);
            }
            g->ab_host = ab;
            if ((ce = upload(&g->ab, ab, st)) != cudaSuccess) goto cuda_fail;
            if ((ce = upload(&g->ab_ph, abp, st)) != cudaSuccess) goto cuda_fail;
        }
        if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) goto cuda_fail;
    } else {
        // ---- REF_COMPAT: single-precision inputs exactly as the reference
        // wrapper casts them (RCA.m:601-626), tables built on the device ----
        std::vector<float> rku((size_t)n_rxkey), rkz((size_t)n_rxkey), tkv((size_t)n_txkey), tkz((size_t)n_txkey);
        for (int64_t k = 0; k < n_rxkey; ++k) { rku[k] = (float)rk_u(k); rkz[k] = (float)k_z(k); }
        for (int64_t k = 0; k < n_txkey; ++k) { tkv[k] = (float)tk_v(k); tkz[k] = (float)k_z(k); }
        std::vector<float> eu((size_t)ne), ezf((size_t)ne), vu((size_t)nt), vv((size_t)nt), vz((size_t)nt), md((size_t)nt);
        for (int64_t r = 0; r < ne; ++r) { eu[r] = (float)ele_u[r]; ezf[r] = (float)ez[r]; }
        for (int64_t t = 0; t < nt; ++t) {
            vu[t] = (float)vs_u[t]; vv[t] = (float)vs_v[t]; vz[t] = (float)g->vs_z[t]; md[t] = (float)g->min_dist[t];
        }
        float *buf = nullptr;
        const size_t nf = rku.size() + rkz.size() + tkv.size() + tkz.size() + eu.size() + ezf.size() + 4 * nt;
        if ((ce = cudaMalloc(&buf, nf * sizeof(float))) != cudaSuccess) goto cuda_fail;
        {
            size_t off = 0;
            auto put = [&](const std::vector<float> &v) {
                float *p = buf + off;
                cudaMemcpyAsync(p, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice, st);
                off += v.size();
                return (const float *)p;
            };
            RefTableParams p{};
            p.rx_key_u = put(rku); p.rx_key_z = put(rkz); p.tx_key_v = put(tkv); p.tx_key_z = put(tkz);
            p.ele_u = put(eu); p.ele_z = put(ezf);
            p.vs_u = put(vu); p.vs_v = put(vv); p.vs_z = put(vz); p.min_dist = put(md);
            p.n_rxkey = n_rxkey; p.n_txkey = n_txkey; p.n_ele = (int)ne; p.n_tx = (int)nt;
            const float apx = (float)g->ap_x, apy = (float)g->ap_y;
            p.half_ap_u = (float)(0.5 * (double)(rxx ? apx : apy));
            p.half_ap_v = (float)(0.5 * (double)(rxx ? apy : apx));
            p.ap_z = (float)g->ap_z;
            p.fnumber = (float)g->fnumber;
            p.inv_c = 1.0f / (float)g->c;
            p.receive_x = rxx ? 1 : 0;
            p.mask_transmit = g->mask_transmit;
            ce = cudaMalloc(&g->rx_tab, sizeof(float4) * ne * n_rxkey);
            if (ce == cudaSuccess) ce = cudaMalloc(&g->tx_tab, sizeof(float4) * nt * n_txkey);
            if (ce == cudaSuccess) ce = cudaMalloc(&g->apod_sum, sizeof(float) * n_rxkey);
            if (ce == cudaSuccess && g->mask_transmit) ce = cudaMalloc(&g->cone_u, (size_t)(nt * n_rxkey));
            float *ratio_d = nullptr;
            if (ce == cudaSuccess) ce = cudaMalloc(&ratio_d, sizeof(float));
            if (ce == cudaSuccess) {
                p.rx_tab = g->rx_tab; p.tx_tab = g->tx_tab; p.apod_sum = g->apod_sum; p.cone_u = g->cone_u;
                p.ratio_out = ratio_d;
                p.fd = (float)g->fd; p.fs = (float)g->fs;
                ce = launch_ref_tables(p, st);
            }
            std::vector<float4> rxh, txh;
            float ratio = 0.f;
            if (ce == cudaSuccess) {
                rxh.resize((size_t)(ne * n_rxkey));
                txh.resize((size_t)(nt * n_txkey));
                ce = cudaMemcpyAsync(rxh.data(), g->rx_tab, rxh.size() * sizeof(float4), cudaMemcpyDeviceToHost, st);
                if (ce == cudaSuccess)
                    ce = cudaMemcpyAsync(txh.data(), g->tx_tab, txh.size() * sizeof(float4), cudaMemcpyDeviceToHost, st);
                if (ce == cudaSuccess)
                    ce = cudaMemcpyAsync(&ratio, ratio_d, sizeof(float), cudaMemcpyDeviceToHost, st);
                if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
            }
            cudaFree(ratio_d);
            cudaFree(buf);
            if (ce != cudaSuccess) goto cuda_fail;
            for (size_t i = 0; i < rxh.size(); ++i)
                g->rx_delay[i] = rxh[i].z != 0.0f ? (float)(rxh[i].x * g->fs) : NAN;
            for (size_t i = 0; i < txh.size(); ++i) g->tx_delay[i] = (float)(txh[i].x * g->fs);
            g->ref.fs = (float)g->fs;
            g->ref.fd = (float)g->fd;
            g->ref.t0 = (float)g->t0;
            g->ref.inv_c = p.inv_c;
            g->ref.ratio = ratio;
        }
        if (d->ab_law) {
            const int64_t n_ab = d->ab_per_tx ? nt * ne : ne;
            std::vector<float> ab((size_t)n_ab);
            for (int64_t i = 0; i < n_ab; ++i) ab[i] = (float)d->ab_law[i];
            g->ab_host.resize((size_t)n_ab);
            for (int64_t i = 0; i < n_ab; ++i) g->ab_host[i] = (float)(d->ab_law[i] * g->fs);
            if ((ce = upload(&g->ab, ab, st)) != cudaSuccess) goto cuda_fail;
            if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) goto cuda_fail;
        }
    }
    if (mode == MODE_EXACT && kind != K_QUAD3) {
        std::vector<float> wt = weight_table(kind);
        if ((ce = upload(&g->wtab, wt, st)) != cudaSuccess) goto cuda_fail;
        if ((ce = cudaStreamSynchronize(st)) != cudaSuccess) goto cuda_fail;
    }
    g->has_ab = d->ab_law ? 1 : 0;
    g->ab_per_tx = d->ab_per_tx ? 1 : 0;
    *out = g.release();
    return RCABF_OK;

cuda_fail:
    free_geometry(g.release());
    (void)ce;
    return RCABF_ERR_CUDA;
}

}  // namespace rcabf

rcabf::DevGeom rcabf_geometry::dev() const
{
    rcabf::DevGeom d{};
    d.rx_tab = rx_tab; d.tx_tab = tx_tab; d.cone_u = cone_u; d.apod_sum = apod_sum;
    d.ab = ab; d.ab_ph = ab_ph; d.ab_per_tx = ab_per_tx; d.mode = mode;
    d.wtab = wtab;
    d.n_ele = n_ele; d.n_tx = n_tx;
    d.n_z = n_z; d.n_u = n_u; d.n_v = n_v; d.s_z = s_z; d.s_u = s_u; d.s_v = s_v; d.n_pix = n_pix;
    d.ref = ref;
    return d;
}

int rcabf_geometry::window_rows(const rcabf::TileShape &ts)
{
    std::lock_guard<std::mutex> lk(mu);
    auto it = spreads.find(ts);
    if (it == spreads.end()) {
        rcabf::TileSpread sp;
        const int64_t tiles_z = (n_z + ts.tz - 1) / ts.tz;
        const int64_t tiles_u = (n_u + ts.tu - 1) / ts.tu;
        const int64_t tiles_v = (n_v + ts.tv - 1) / ts.tv;
        sp.rx_spread.assign((size_t)tiles_z, 0.f);
        sp.tx_spread.assign((size_t)tiles_z, 0.f);
        auto scan = [&](const std::vector<float> &tab, int64_t rows, int64_t n_a, int64_t ta, int64_t tiles_a,
                        std::vector<float> &outv) {
            for (int64_t r = 0; r < rows; ++r)
                for (int64_t a0 = 0; a0 < tiles_a; ++a0)
                    for (int64_t z0 = 0; z0 < tiles_z; ++z0) {
                        float lo = INFINITY, hi = -INFINITY;
                        for (int64_t a = a0 * ta; a < std::min(n_a, (a0 + 1) * ta); ++a)
                            for (int64_t z = z0 * ts.tz; z < std::min(n_z, (z0 + 1) * ts.tz); ++z) {
                                const float v = tab[(size_t)(r * n_a * n_z + a * n_z + z)];
                                if (std::isnan(v)) continue;
                                lo = std::min(lo, v);
                                hi = std::max(hi, v);
                            }
                        if (hi >= lo) outv[(size_t)z0] = std::max(outv[(size_t)z0], hi - lo);
                    }
        };
        scan(rx_delay, n_ele, n_u, ts.tu, tiles_u, sp.rx_spread);
        scan(tx_delay, n_tx, n_v, ts.tv, tiles_v, sp.tx_spread);
        it = spreads.emplace(ts, std::move(sp)).first;
    }
    float m = 0.f;
    for (size_t i = 0; i < it->second.rx_spread.size(); ++i)
        m = std::max(m, it->second.rx_spread[i] + it->second.tx_spread[i]);
    return (int)std::ceil(m) + rcabf::kind_taps(kind) + 3;
}

int64_t rcabf_geometry::tc_chunks(const rcabf::TileShape &ts, int64_t n_sample)
{
    std::lock_guard<std::mutex> lk(mu);
    const std::array<int64_t, 3> key{ts.tu, ts.tv, n_sample};
    auto it = tc_chunk_counts.find(key);
    if (it != tc_chunk_counts.end()) return it->second;
    const int64_t tiles_u = (n_u + ts.tu - 1) / ts.tu, tiles_v = (n_v + ts.tv - 1) / ts.tv;
    const int lo_taps = rcabf::kind_lo(kind), taps = rcabf::kind_taps(kind);
    // per (element, u tile, z) and (transmit, v tile, z): min / max table delay
    // of the valid entries (as the window-range kernel forms them)
    auto ranges = [&](const std::vector<float> &tab, int64_t rows, int64_t n_a, int64_t ta, int64_t tiles_a,
                      std::vector<float> &mn, std::vector<float> &mx) {
        mn.assign((size_t)(rows * tiles_a * n_z), INFINITY);
        mx.assign((size_t)(rows * tiles_a * n_z), -INFINITY);
        for (int64_t r = 0; r < rows; ++r)
            for (int64_t a = 0; a < n_a; ++a)
                for (int64_t z = 0; z < n_z; ++z) {
                    const float v = tab[(size_t)(r * n_a * n_z + a * n_z + z)];
                    if (std::isnan(v)) continue;
                    const size_t o = (size_t)((r * tiles_a + a / ta) * n_z + z);
                    mn[o] = std::min(mn[o], v);
                    mx[o] = std::max(mx[o], v);
                }
    };
    std::vector<float> rmn, rmx, tmn, tmx;
    ranges(rx_delay, n_ele, n_u, ts.tu, tiles_u, rmn, rmx);
    ranges(tx_delay, n_tx, n_v, ts.tv, tiles_v, tmn, tmx);
    int64_t total = 0;
    const float fmax_n = (float)n_sample;
    for (int64_t t = 0; t < n_tx; ++t)
        for (int64_t e = 0; e < n_ele; ++e) {
            const float ab = ab_host.empty() ? 0.0f : ab_host[(size_t)(ab_per_tx ? t * n_ele + e : e)];
            for (int64_t tu = 0; tu < tiles_u; ++tu)
                for (int64_t z = 0; z < n_z; ++z) {
                    const size_t ro = (size_t)((e * tiles_u + tu) * n_z + z);
                    if (!(rmn[ro] <= rmx[ro])) continue;
                    for (int64_t tv = 0; tv < tiles_v; ++tv) {
                        const size_t to = (size_t)((t * tiles_v + tv) * n_z + z);
                        if (!(tmn[to] <= tmx[to])) continue;
                        volatile float l0 = tmn[to] + rmn[ro];
                        volatile float h0 = tmx[to] + rmx[ro];
                        float lo_f = l0 + ab, hi_f = h0 + ab;
                        lo_f = std::min(std::max(std::floor(lo_f), -1.0f), fmax_n);
                        hi_f = std::min(std::max(std::floor(hi_f), -1.0f), fmax_n);
                        const int l = std::max((int)lo_f - lo_taps, 0);
                        const int h = std::min((int)hi_f - lo_taps + taps - 1, (int)n_sample - 2);
                        if (h < l) continue;
                        const int nk = (h - l + 1 + 15) / 16;
                        if (nk <= rcabf::TC_MAX_ROWS / 16) total += nk;
                    }
                }
        }
    tc_chunk_counts[key] = total;
    return total;
}

int rcabf_geometry::vb_shift(int block)
{
    std::lock_guard<std::mutex> lk(mu);
    auto it = vb_shifts.find(block);
    if (it != vb_shifts.end()) return it->second;
    int d = -1;
    if (mode == rcabf::MODE_EXACT && grid_kind == RCABF_GRID_RECTILINEAR && n_v >= 2) {
        // The voxels of a block share the receive part of the index (and the
        // aberration shift), so floor(itx_v + r) - floor(itx_w + r) is at
        // most ceil(|itx_v - itx_w|); a margin covers the float sums.
        float spread = 0.f;
        for (int64_t t = 0; t < n_tx; ++t)
            for (int64_t v0 = 0; v0 < n_v; v0 += block)
                for (int64_t z = 0; z < n_z; ++z) {
                    float lo = INFINITY, hi = -INFINITY;
                    for (int64_t v = v0; v < std::min(n_v, v0 + block); ++v) {
                        const float x = tx_delay[(size_t)((t * n_v + v) * n_z + z)];
                        lo = std::min(lo, x);
                        hi = std::max(hi, x);
                    }
                    spread = std::max(spread, hi - lo);
                }
        d = (int)std::ceil(spread + 1e-3f);
        if (d < 1) d = 1;
    }
    vb_shifts[block] = d;
    return d;
}
