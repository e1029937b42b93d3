// Generated by gen_weight_poly.py -- do not edit.
// Degree-8 polynomials in u = 2d - 1 of the left-hand interpolation
// weights w_j(d), j < TAPS/2; w_{TAPS-1-j}(d) = w_j at -u.
// Coefficients live in constant memory (uniform operands of the FMAs).
#pragma once

namespace rcabf {

constexpr int WPOLY_DEG = 8;

template <int KIND> struct WeightPoly;

// K_REF6: max fit error 1.12e-06
static __constant__ float WPOLY_K_REF6[3][9] = {
    {-2.292635400e-02f, -8.836707306e-03f, 3.980600346e-02f, 8.510068191e-03f, -1.988748774e-02f, 6.549056671e-04f, 3.221626419e-03f, -3.286282217e-04f, -2.138384259e-04f},
    {-6.368437609e-02f, 9.247301927e-02f, 4.363743636e-02f, -1.062029447e-01f, 2.455305960e-02f, 1.457026981e-02f, -4.860630306e-03f, -8.406574259e-04f, 3.546052027e-04f},
    {5.731591807e-01f, -6.961574710e-01f, -6.472297458e-02f, 2.239244632e-01f, -1.063087087e-02f, -2.981932153e-02f, 2.372569549e-03f, 2.053395512e-03f, -1.779537914e-04f}};
template <> struct WeightPoly<K_REF6> {
    static constexpr int HALF = 3;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY_K_REF6[j][m]; }
};

// K_LANCZOS2: max fit error 1.12e-06
static __constant__ float WPOLY_K_LANCZOS2[2][9] = {
    {-6.368437609e-02f, 9.247301927e-02f, 4.363743636e-02f, -1.062029447e-01f, 2.455305960e-02f, 1.457026981e-02f, -4.860630306e-03f, -8.406574259e-04f, 3.546052027e-04f},
    {5.731591807e-01f, -6.961574710e-01f, -6.472297458e-02f, 2.239244632e-01f, -1.063087087e-02f, -2.981932153e-02f, 2.372569549e-03f, 2.053395512e-03f, -1.779537914e-04f}};
template <> struct WeightPoly<K_LANCZOS2> {
    static constexpr int HALF = 2;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY_K_LANCZOS2[j][m]; }
};

// K_LANCZOS3: max fit error 4.88e-07
static __constant__ float WPOLY_K_LANCZOS3[3][9] = {
    {2.431709069e-02f, -3.177962398e-02f, -2.159438587e-02f, 3.811809119e-02f, -4.025457159e-03f, -6.743619638e-03f, 1.409867822e-03f, 4.052975720e-04f, -1.071416215e-04f},
    {-1.350949172e-01f, 9.006240410e-02f, 1.401538636e-01f, -1.034299220e-01f, -4.152389678e-03f, 1.420981639e-02f, -9.953854842e-04f, -8.426428615e-04f, 8.885136568e-05f},
    {6.079271041e-01f, -6.645240963e-01f, -1.122099433e-01f, 1.835606860e-01f, 3.978657976e-03f, -2.018404076e-02f, 3.384757005e-04f, 1.147930225e-03f, -3.430345598e-05f}};
template <> struct WeightPoly<K_LANCZOS3> {
    static constexpr int HALF = 3;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY_K_LANCZOS3[j][m]; }
};

// K_LANCZOS4: max fit error 3.24e-07
static __constant__ float WPOLY_K_LANCZOS4[4][9] = {
    {-1.266088060e-02f, 1.562042682e-02f, 1.239145835e-02f, -1.897269799e-02f, 7.389239865e-04f, 3.590260956e-03f, -5.133529177e-04f, -2.380817188e-04f, 4.386216033e-05f},
    {5.990948595e-02f, -3.370828630e-02f, -6.744278285e-02f, 4.059144974e-02f, 7.415177655e-03f, -7.345860702e-03f, 1.534183975e-04f, 4.628797843e-04f, -3.530932229e-05f},
    {-1.664152334e-01f, 8.387349510e-02f, 1.807127884e-01f, -9.569334900e-02f, -1.448763804e-02f, 1.252212683e-02f, 1.694021416e-04f, -7.025411724e-04f, 2.068797774e-05f},
    {6.203830139e-01f, -6.526052374e-01f, -1.283732447e-01f, 1.686102986e-01f, 8.130628343e-03f, -1.687146911e-02f, -1.339791538e-04f, 8.667293713e-04f, -6.420909172e-06f}};
template <> struct WeightPoly<K_LANCZOS4> {
    static constexpr int HALF = 4;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY_K_LANCZOS4[j][m]; }
};

}  // namespace rcabf
