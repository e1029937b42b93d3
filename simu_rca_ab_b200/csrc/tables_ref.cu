// REF_COMPAT delay tables: the reference kernel's single-precision delay,
// apodisation and transmit-cone arithmetic (RCA.cu:85-98, 153-174, 190-219,
// 255-311), evaluated once per table key on the device with CUDA's own math
// functions.  Compiled with -fmad=false and no fast math: every expression
// below rounds exactly where the C source of the reference rounds.
#include <cuda_runtime.h>

#include "launchers.h"

namespace rcabf {

#define REF_PI_F 3.14159265358979323846f

// RCA.cu:85-98 (differences in float, products in double, arccosine in float).
__device__ float ref_angle_aperture(float ax, float ay, float bx, float by, float cx, float cy)
{
    double abx = bx - ax;
    double aby = by - ay;
    double acx = cx - ax;
    double acy = cy - ay;
    return acosf(((abx * acx) + (aby * acy)) * rsqrt((abx * abx + aby * aby) * (acx * acx + acy * acy)));
}

// Half of the transmit-cone test of RCA.cu:193-214 along one lateral axis:
// the pixel at lateral coordinate p (depth z) lies inside the cone from the
// virtual source (vl, vz) through the aperture edges (+-h, -az).
__device__ bool ref_cone_half(float vl, float vz, float h, float az, float p, float z)
{
    const float cone = ref_angle_aperture(vl, vz, -h, -az, h, -az);
    return ref_angle_aperture(vl, vz, -h, -az, p, z) <= cone &&
           ref_angle_aperture(vl, vz, h, -az, p, z) <= cone;
}

__global__ void ref_rx_table_kernel(const RefTableParams p)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)p.n_ele * p.n_rxkey) return;
    const int64_t k = i % p.n_rxkey;
    const int r = (int)(i / p.n_rxkey);
    const float pu = p.rx_key_u[k], pz = p.rx_key_z[k];
    const float aperture_f = pz / p.fnumber;                       // RCA.cu:174
    const float aperture = fabsf(pu - p.ele_u[r]);                 // RCA.cu:286/290
    const bool valid = aperture < aperture_f;                      // RCA.cu:294
    float apod = 0.0f;
    if (valid) apod = 0.5 * (1 + cospif(fdividef(aperture, aperture_f)));  // RCA.cu:299
    const float delay_rx = hypotf(aperture, pz - p.ele_z[r]) * p.inv_c;   // RCA.cu:308-309
    p.rx_tab[i] = make_float4(delay_rx, apod, valid ? 1.0f : 0.0f, 0.0f);
}

// Sum of the apodisation over elements in element order (RCA.cu:301-304).
__global__ void ref_apod_sum_kernel(const RefTableParams p)
{
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= p.n_rxkey) return;
    float m = 0.0f;
    for (int r = 0; r < p.n_ele; ++r) {
        const float4 e = p.rx_tab[(int64_t)r * p.n_rxkey + k];
        if (e.z != 0.0f) m += e.y;
    }
    p.apod_sum[k] = m;
}

__global__ void ref_tx_table_kernel(const RefTableParams p)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)p.n_tx * p.n_txkey) return;
    const int64_t k = i % p.n_txkey;
    const int t = (int)(i / p.n_txkey);
    const float pv = p.tx_key_v[k], pz = p.tx_key_z[k];
    float delay_tx;
    // RCA.cu:256-269: the coordinate along the receive axis is multiplied by
    // zero; the norm of (+-0, a, b) equals the norm of (0, a, b).
    if (p.receive_x)
        delay_tx = (norm3df(0.0f, pv - p.vs_v[t], pz - p.vs_z[t]) - p.min_dist[t]) * p.inv_c;
    else
        delay_tx = (norm3df(pv - p.vs_v[t], 0.0f, pz - p.vs_z[t]) - p.min_dist[t]) * p.inv_c;
    bool cone = true;
    if (p.mask_transmit) cone = ref_cone_half(p.vs_v[t], p.vs_z[t], p.half_ap_v, p.ap_z, pv, pz);
    p.tx_tab[i] = make_float4(delay_tx, cone ? 1.0f : 0.0f, pz, 0.0f);
}

__global__ void ref_cone_u_kernel(const RefTableParams p)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (int64_t)p.n_tx * p.n_rxkey) return;
    const int64_t k = i % p.n_rxkey;
    const int t = (int)(i / p.n_rxkey);
    p.cone_u[i] = ref_cone_half(p.vs_u[t], p.vs_z[t], p.half_ap_u, p.ap_z, p.rx_key_u[k], p.rx_key_z[k]) ? 1 : 0;
}

__global__ void ref_scalar_kernel(const RefTableParams p)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *p.ratio_out = fdividef(p.fd, p.fs);  // RCA.cu:372
}

cudaError_t launch_ref_tables(const RefTableParams &p, cudaStream_t st)
{
    const int B = 256;
    ref_scalar_kernel<<<1, 32, 0, st>>>(p);
    const int64_t n_rx = (int64_t)p.n_ele * p.n_rxkey, n_tx = (int64_t)p.n_tx * p.n_txkey;
    ref_rx_table_kernel<<<(unsigned)((n_rx + B - 1) / B), B, 0, st>>>(p);
    ref_apod_sum_kernel<<<(unsigned)((p.n_rxkey + B - 1) / B), B, 0, st>>>(p);
    ref_tx_table_kernel<<<(unsigned)((n_tx + B - 1) / B), B, 0, st>>>(p);
    if (p.mask_transmit && p.cone_u) {
        const int64_t n_c = (int64_t)p.n_tx * p.n_rxkey;
        ref_cone_u_kernel<<<(unsigned)((n_c + B - 1) / B), B, 0, st>>>(p);
    }
    return cudaGetLastError();
}

}  // namespace rcabf
