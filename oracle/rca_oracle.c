/*
 * oracle/rca_oracle.c -- TEST INFRASTRUCTURE ONLY.  Nothing in the product
 * links or calls this file; tests/, __graft_entry__.smoke() and bench.py's
 * accuracy/CPU-baseline legs use it as the checker.
 *
 * A plain-C restatement of the reference row-column-array (RCA) delay-and-sum
 * I/Q beamformer kernel
 *     MATLAB/lib/beamformer/RCA/bfVirtualSourceGeneric_RCA.cu:103-390
 * in two arithmetic modes:
 *
 *   oracle_rca_fp32ref : the reference's own single-precision arithmetic,
 *       operation for operation (same association, same float/double
 *       promotions), with the transcendental functions of refmath.h.  On the
 *       CPU it must agree bit-for-bit with the reference kernel source built
 *       by oracle/ref_cpu_harness.cpp; tests/test_oracle_pin.py checks that.
 *
 *   oracle_rca_fp64 : the same delay-and-sum model evaluated in double
 *       precision from double inputs (no FP32 cancellation in the transmit
 *       delay), with three interpolation kernels: the reference's quadratic
 *       (3 taps), the reference's 6-tap sinc(x)*sinc(x/2), and Lanczos-a
 *       (2a taps, window sinc(x/a)).  This is the accuracy oracle for the
 *       CUDA path's exact-table mode.
 *
 * Layouts follow the reference kernel:
 *   data   : [frame][tx][channel][sample] complex, interleaved (re, im)
 *   dataBf : [frame][tx][pixel] complex, interleaved   (per transmit)
 *            or [channel][frame][tx][pixel] when per_channel is set
 *            (the NoSum variants, NoSum/bfVirtualSourceGeneric_RCA_Nosum.cu:228-229, 376-383)
 *   mask   : [tx][pixel]
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "refmath.h"

#define ORACLE_API __attribute__((visibility("default")))

/* Interpolation kernels (values shared with the product's C ABI). */
enum { OR_INTERP_QUAD3 = 0, OR_INTERP_REF6 = 1, OR_INTERP_LANCZOS = 2 };

/* ------------------------------------------------------------------------ */
/* FP32 restatement of the reference arithmetic                              */
/* ------------------------------------------------------------------------ */

static const float OR_PI_F = 3.14159265358979323846f; /* RCA.cu:76 */

/* RCA.cu:79-82 */
static inline float or_sinc_f(float x)
{
    float r = rm_fdividef(rm_sinpif(x), OR_PI_F * x);
    return fminf(r, 1.0f);
}

/* RCA.cu:85-98: angle between AB and AC.  The differences are formed in
 * float (float operands), the rest in double, the arccosine in float. */
static inline float or_angle_aperture_f(float ax, float ay, float bx, float by,
                                        float cx, float cy)
{
    double abx = (double)(bx - ax);
    double aby = (double)(by - ay);
    double acx = (double)(cx - ax);
    double acy = (double)(cy - ay);
    double num = (abx * acx) + (aby * acy);
    double den = (abx * abx + aby * aby) * (acx * acx + acy * acy);
    return rm_acosf((float)(num * rm_rsqrt(den)));
}

/* RCA.cu:190-219 */
static inline int or_mask_transmit_f(float vx, float vy, float vz, float hx,
                                     float hy, float az, float px, float py,
                                     float pz)
{
    float cone_x = or_angle_aperture_f(vx, vz, -hx, -az, hx, -az);
    float cone_y = or_angle_aperture_f(vy, vz, -hy, -az, hy, -az);
    return or_angle_aperture_f(vx, vz, -hx, -az, px, pz) <= cone_x &&
           or_angle_aperture_f(vx, vz, hx, -az, px, pz) <= cone_x &&
           or_angle_aperture_f(vy, vz, -hy, -az, py, pz) <= cone_y &&
           or_angle_aperture_f(vy, vz, hy, -az, py, pz) <= cone_y;
}

typedef struct {
    const float *gx, *gy, *gz;      /* per pixel */
    const float *ex, *ey, *ez;      /* per channel (centred) */
    const float *vsx, *vsy, *vsz;   /* per transmit */
    const float *min_dist;          /* per transmit */
    const float *ab_law;            /* NULL, [channel] or [tx][channel] (s) */
    int ab_per_tx;
    int receive_x;
    float ap_x, ap_y, ap_z;
    float fs, fd, c, t0, fnumber;
    int64_t n_pix, n_ch, n_tx, n_frame, n_sample;
    int lanczos;                    /* 1: 6-tap, 0: quadratic */
    int mask_transmit;
    int per_channel;                /* NoSum layout, assignment instead of sum */
} or_args32;

/* One (pixel, transmit, frame) of RCA.cu:149-383. */
static void or_pixel_f(const or_args32 *a, const float *data, float *out,
                       float *mask, int64_t p, int64_t t, int64_t f)
{
    const float px = a->gx[p], py = a->gy[p], pz = a->gz[p];
    const float vx = a->vsx[t], vy = a->vsy[t], vz = a->vsz[t];
    const float md = a->min_dist[t];
    const float inv_c = 1.0f / a->c;                       /* RCA.cu:164 */
    const float half_x = (float)(0.5 * (double)a->ap_x);   /* RCA.cu:172 */
    const float half_y = (float)(0.5 * (double)a->ap_y);   /* RCA.cu:173 */
    const float ap_f = pz / a->fnumber;                    /* RCA.cu:174 */

    if (a->mask_transmit &&
        !or_mask_transmit_f(vx, vy, vz, half_x, half_y, a->ap_z, px, py, pz))
        return;                                            /* RCA.cu:224 */

    const int lo = a->lanczos ? 2 : 1, hi = a->lanczos ? 3 : 1; /* RCA.cu:234-243 */
    const int64_t pix_tx = p + t * a->n_pix;
    const int64_t n_ptf = a->n_pix * a->n_tx * a->n_frame;
    const int64_t o = 2 * (p + t * a->n_pix + f * a->n_pix * a->n_tx);

    if (f == 0) mask[pix_tx] = 0.0f;                       /* RCA.cu:247-250 */
    if (!a->per_channel) { out[o] = 0.0f; out[o + 1] = 0.0f; }

    float delay_tx;                                        /* RCA.cu:256-269 */
    if (a->receive_x)
        delay_tx = (rm_norm3df((px - vx) * 0.0f, py - vy, pz - vz) - md) * inv_c;
    else
        delay_tx = (rm_norm3df(px - vx, (py - vy) * 0.0f, pz - vz) - md) * inv_c;

    const float ratio = rm_fdividef(a->fd, a->fs);
    for (int64_t ch = 0; ch < a->n_ch; ++ch) {             /* RCA.cu:273 */
        float *acc = a->per_channel ? out + o + 2 * ch * n_ptf : out + o;
        if (a->per_channel) { acc[0] = 0.0f; acc[1] = 0.0f; }
        const float ex = a->ex[ch], ey = a->ey[ch], ez = a->ez[ch];
        const float ap = a->receive_x ? fabsf(px - ex) : fabsf(py - ey);
        if (!(ap < ap_f)) continue;                        /* RCA.cu:294 */
        float apod = (float)(0.5 * (double)(1.0f + rm_cospif(rm_fdividef(ap, ap_f))));
        if (f == 0) mask[pix_tx] += apod;                  /* RCA.cu:301-304 */
        float delay_rx = rm_hypotf(ap, pz - ez) * inv_c;   /* RCA.cu:308-309 */
        if (a->ab_law)
            delay_rx = a->ab_law[a->ab_per_tx ? t * a->n_ch + ch : ch] + delay_rx;
        const float idx = (delay_tx + delay_rx + a->t0) * a->fs; /* RCA.cu:310-311 */
        const int64_t base = 2 * (ch * a->n_sample + t * a->n_sample * a->n_ch +
                                  f * a->n_sample * a->n_ch * a->n_tx);
        const int n0 = (int)floorf(idx);                   /* RCA.cu:319 */
        if (!(n0 >= lo && n0 < a->n_sample - 1 - hi)) continue; /* RCA.cu:323 */
        const float d = idx - (float)n0;                   /* RCA.cu:325 */
        const float *s = data + base + 2 * (int64_t)n0;
        float re, im;
        if (a->lanczos) {                                  /* RCA.cu:331-350 */
            float q[6];
            for (int k = 0; k < 6; ++k) {
                float x = d + (float)(2 - k);
                q[k] = or_sinc_f(x) * or_sinc_f(x / 2.0f);
            }
            re = q[0] * s[-4] + q[1] * s[-2] + q[2] * s[0] + q[3] * s[2] + q[4] * s[4] + q[5] * s[6];
            im = q[0] * s[-3] + q[1] * s[-1] + q[2] * s[1] + q[3] * s[3] + q[4] * s[5] + q[5] * s[7];
        } else {                                           /* RCA.cu:355-365 */
            const float q0 = d * (d - 1.0f) / 2.0f;
            const float q1 = -(d - 1.0f) * (d + 1.0f);
            const float q2 = d * (d + 1.0f) / 2.0f;
            re = q0 * s[-2] + q1 * s[0] + q2 * s[2];
            im = q0 * s[-1] + q1 * s[1] + q2 * s[3];
        }
        /* RCA.cu:371-380 */
        const float delta = -2.0f * OR_PI_F * idx * ratio + 4.0f * OR_PI_F * a->fd * pz * inv_c;
        const float cs = rm_cosf(delta), sn = rm_sinf(delta);
        if (a->per_channel) {
            acc[0] = apod * (re * cs + im * sn);
            acc[1] = apod * (-re * sn + im * cs);
        } else {
            acc[0] += apod * (re * cs + im * sn);
            acc[1] += apod * (-re * sn + im * cs);
        }
    }
}

ORACLE_API int oracle_rca_fp32ref(
    float *dataBf, float *mask, const float *data,
    const float *gx, const float *gy, const float *gz,
    const float *ex, const float *ey, const float *ez,
    const float *vsx, const float *vsy, const float *vsz, const float *min_dist,
    int receive_x, float ap_x, float ap_y, float ap_z,
    float fs, float fd, float c, float t0, float fnumber,
    int64_t n_pix, int64_t n_ch, int64_t n_tx, int64_t n_frame, int64_t n_sample,
    int lanczos, int mask_transmit, int per_channel,
    const float *ab_law, int ab_per_tx, int n_threads)
{
    if (n_pix <= 0 || n_ch <= 0 || n_tx <= 0 || n_frame <= 0 || n_sample <= 0) return 1;
    or_args32 a = {gx, gy, gz, ex, ey, ez, vsx, vsy, vsz, min_dist, ab_law, ab_per_tx,
                   receive_x, ap_x, ap_y, ap_z, fs, fd, c, t0, fnumber,
                   n_pix, n_ch, n_tx, n_frame, n_sample, lanczos, mask_transmit,
                   per_channel};
    const int64_t n_items = n_frame * n_tx;
    if (n_threads <= 0) n_threads = 1;
    /* Frame 0 owns the mask writes; every (pixel, tx, frame) is independent. */
#pragma omp parallel for collapse(2) schedule(static) num_threads(n_threads)
    for (int64_t it = 0; it < n_items; ++it)
        for (int64_t p = 0; p < n_pix; ++p)
            or_pixel_f(&a, data, dataBf, mask, p, it % n_tx, it / n_tx);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* FP64 delay-and-sum (accuracy oracle)                                      */
/* ------------------------------------------------------------------------ */

static inline double or_sinc_d(double x)
{
    if (x == 0.0) return 1.0;
    return sin(M_PI * x) / (M_PI * x);
}

/* Interpolation weights for fractional offset d in [0, 1).  Tap j sits on
 * sample n0 - lo + j.  Returns the tap count. */
static int or_weights_d(int interp, int a, double d, double *w, int *lo_out, int *hi_out)
{
    if (interp == OR_INTERP_QUAD3) {                       /* RCA.cu:355-357 */
        w[0] = d * (d - 1.0) / 2.0;
        w[1] = -(d - 1.0) * (d + 1.0);
        w[2] = d * (d + 1.0) / 2.0;
        *lo_out = 1; *hi_out = 1;
        return 3;
    }
    if (interp == OR_INTERP_REF6) {                        /* RCA.cu:331-336 */
        for (int j = 0; j < 6; ++j) {
            double x = d - (double)(j - 2);
            w[j] = or_sinc_d(x) * or_sinc_d(x / 2.0);
        }
        *lo_out = 2; *hi_out = 3;
        return 6;
    }
    /* Lanczos-a: L(x) = sinc(x) sinc(x/a), |x| < a, taps n0-a+1 .. n0+a. */
    for (int j = 0; j < 2 * a; ++j) {
        double x = d - (double)(j - (a - 1));
        w[j] = (fabs(x) < (double)a) ? or_sinc_d(x) * or_sinc_d(x / (double)a) : 0.0;
    }
    *lo_out = a - 1; *hi_out = a;
    return 2 * a;
}

/* data64: [frame][tx][ch][sample] complex128 interleaved, or (data32 != NULL)
 * the same layout in complex64, read and promoted to double. */
ORACLE_API int oracle_rca_fp64(
    double *dataBf, double *mask, const double *data64, const float *data32,
    const double *gx, const double *gy, const double *gz,
    const double *ex, const double *ey, const double *ez,
    const double *vsx, const double *vsy, const double *vsz, const double *min_dist,
    int receive_x, double ap_x, double ap_y, double ap_z,
    double fs, double fd, double c, double t0, double fnumber,
    int64_t n_pix, int64_t n_ch, int64_t n_tx, int64_t n_frame, int64_t n_sample,
    int interp, int lanczos_a, int mask_transmit, int per_channel,
    const double *ab_law, int ab_per_tx, int n_threads)
{
    if (n_pix <= 0 || n_ch <= 0 || n_tx <= 0 || n_frame <= 0 || n_sample <= 0) return 1;
    if (interp == OR_INTERP_LANCZOS && (lanczos_a < 1 || lanczos_a > 16)) return 2;
    if ((data64 == NULL) == (data32 == NULL)) return 3;
    const int64_t n_ptf = n_pix * n_tx * n_frame;
    const int64_t n_items = n_frame * n_tx;
    if (n_threads <= 0) n_threads = 1;
#pragma omp parallel for collapse(2) schedule(static) num_threads(n_threads)
    for (int64_t it = 0; it < n_items; ++it) {
        for (int64_t p = 0; p < n_pix; ++p) {
            const int64_t t = it % n_tx, f = it / n_tx;
            const double px = gx[p], py = gy[p], pz = gz[p];
            const double vx = vsx[t], vy = vsy[t], vz = vsz[t];
            const int64_t o = 2 * (p + t * n_pix + f * n_pix * n_tx);
            if (f == 0) mask[p + t * n_pix] = 0.0;
            if (!per_channel) { dataBf[o] = 0.0; dataBf[o + 1] = 0.0; }
            if (mask_transmit) {
                /* RCA.cu:190-214 in double: inside the cone from the virtual
                 * source through both aperture edges, in xz and in yz. */
                const double hx = 0.5 * ap_x, hy = 0.5 * ap_y;
                double ang[6];
                const double P[6][6] = {
                    {vx, vz, -hx, -ap_z, hx, -ap_z}, {vy, vz, -hy, -ap_z, hy, -ap_z},
                    {vx, vz, -hx, -ap_z, px, pz},    {vx, vz, hx, -ap_z, px, pz},
                    {vy, vz, -hy, -ap_z, py, pz},    {vy, vz, hy, -ap_z, py, pz}};
                for (int q = 0; q < 6; ++q) {
                    double abx = P[q][2] - P[q][0], aby = P[q][3] - P[q][1];
                    double acx = P[q][4] - P[q][0], acy = P[q][5] - P[q][1];
                    double cs = (abx * acx + aby * acy) /
                                sqrt((abx * abx + aby * aby) * (acx * acx + acy * acy));
                    ang[q] = acos(fmax(-1.0, fmin(1.0, cs)));
                }
                if (!(ang[2] <= ang[0] && ang[3] <= ang[0] && ang[4] <= ang[1] && ang[5] <= ang[1]))
                    continue;
            }
            double dtx;
            if (receive_x) dtx = (sqrt((py - vy) * (py - vy) + (pz - vz) * (pz - vz)) - min_dist[t]) / c;
            else           dtx = (sqrt((px - vx) * (px - vx) + (pz - vz) * (pz - vz)) - min_dist[t]) / c;
            const double ap_f = pz / fnumber;
            double acc_re = 0.0, acc_im = 0.0;
            for (int64_t ch = 0; ch < n_ch; ++ch) {
                double *pc = per_channel ? dataBf + o + 2 * ch * n_ptf : NULL;
                if (pc) { pc[0] = 0.0; pc[1] = 0.0; }
                const double ap = receive_x ? fabs(px - ex[ch]) : fabs(py - ey[ch]);
                if (!(ap < ap_f)) continue;
                const double apod = 0.5 * (1.0 + cos(M_PI * ap / ap_f));
                if (f == 0) mask[p + t * n_pix] += apod;
                double drx = sqrt(ap * ap + (pz - ez[ch]) * (pz - ez[ch])) / c;
                if (ab_law) drx += ab_law[ab_per_tx ? t * n_ch + ch : ch];
                const double idx = (dtx + drx + t0) * fs;
                const double fl = floor(idx);
                double w[32];
                int lo, hi;
                const int nt = or_weights_d(interp, lanczos_a, idx - fl, w, &lo, &hi);
                if (!(fl >= lo && fl < (double)(n_sample - 1 - hi))) continue;
                const int64_t n0 = (int64_t)fl;
                const int64_t base = 2 * (ch * n_sample + t * n_sample * n_ch +
                                          f * n_sample * n_ch * n_tx) + 2 * (n0 - lo);
                double re = 0.0, im = 0.0;
                for (int j = 0; j < nt; ++j) {
                    double sr = data64 ? data64[base + 2 * j] : (double)data32[base + 2 * j];
                    double si = data64 ? data64[base + 2 * j + 1] : (double)data32[base + 2 * j + 1];
                    re += w[j] * sr;
                    im += w[j] * si;
                }
                /* out += apod * s * exp(-j*delta), delta = -2 pi idx fd/fs + 4 pi fd z / c */
                const double delta = -2.0 * M_PI * idx * fd / fs + 4.0 * M_PI * fd * pz / c;
                const double cs = cos(delta), sn = sin(delta);
                const double vr = apod * (re * cs + im * sn);
                const double vi = apod * (-re * sn + im * cs);
                if (pc) { pc[0] = vr; pc[1] = vi; }
                else { acc_re += vr; acc_im += vi; }
            }
            if (!per_channel) { dataBf[o] = acc_re; dataBf[o + 1] = acc_im; }
        }
    }
    return 0;
}

/* Active-unit count: (pixel, rx, tx) triples inside the f-number aperture and
 * the sample window, per frame.  Used to state the roofline's active work. */
ORACLE_API int64_t oracle_rca_active_units(
    const double *gx, const double *gy, const double *gz,
    const double *ex, const double *ey, const double *ez,
    const double *vsx, const double *vsy, const double *vsz, const double *min_dist,
    int receive_x, double fs, double c, double t0, double fnumber,
    int64_t n_pix, int64_t n_ch, int64_t n_tx, int64_t n_sample, int lo, int hi,
    int n_threads)
{
    int64_t total = 0;
    if (n_threads <= 0) n_threads = 1;
#pragma omp parallel for collapse(2) reduction(+ : total) schedule(static) num_threads(n_threads)
    for (int64_t t = 0; t < n_tx; ++t)
        for (int64_t p = 0; p < n_pix; ++p) {
            const double px = gx[p], py = gy[p], pz = gz[p];
            double dtx = receive_x
                ? (sqrt((py - vsy[t]) * (py - vsy[t]) + (pz - vsz[t]) * (pz - vsz[t])) - min_dist[t]) / c
                : (sqrt((px - vsx[t]) * (px - vsx[t]) + (pz - vsz[t]) * (pz - vsz[t])) - min_dist[t]) / c;
            for (int64_t ch = 0; ch < n_ch; ++ch) {
                const double ap = receive_x ? fabs(px - ex[ch]) : fabs(py - ey[ch]);
                if (!(ap < pz / fnumber)) continue;
                double idx = (dtx + sqrt(ap * ap + (pz - ez[ch]) * (pz - ez[ch])) / c + t0) * fs;
                double fl = floor(idx);
                if (fl >= lo && fl < (double)(n_sample - 1 - hi)) total += 1;
            }
        }
    return total;
}
