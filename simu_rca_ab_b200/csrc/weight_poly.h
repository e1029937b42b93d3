// Generated by gen_weight_poly.py -- do not edit.
// Polynomials in u = 2d - 1 of the left-hand interpolation weights
// w_j(d), j < TAPS/2; w_{TAPS-1-j}(d) = w_j at -u.  Degree 8 for FP32
// sample storage, degree 6 for FP16 / BF16 sample storage.
// Coefficients live in constant memory (uniform operands of the FMAs).
#pragma once

namespace rcabf {

template <int KIND, int DEG> struct WeightPoly;

// K_REF6, degree 8: max fit error 1.12e-06
static __constant__ float WPOLY8_K_REF6[3][9] = {
    {-2.292635400e-02f, -8.836707306e-03f, 3.980600346e-02f, 8.510068191e-03f, -1.988748774e-02f, 6.549056671e-04f, 3.221626419e-03f, -3.286282217e-04f, -2.138384259e-04f},
    {-6.368437609e-02f, 9.247301927e-02f, 4.363743636e-02f, -1.062029447e-01f, 2.455305960e-02f, 1.457026981e-02f, -4.860630306e-03f, -8.406574259e-04f, 3.546052027e-04f},
    {5.731591807e-01f, -6.961574710e-01f, -6.472297458e-02f, 2.239244632e-01f, -1.063087087e-02f, -2.981932153e-02f, 2.372569549e-03f, 2.053395512e-03f, -1.779537914e-04f}};
template <> struct WeightPoly<K_REF6, 8> {
    static constexpr int HALF = 3;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY8_K_REF6[j][m]; }
};

// K_LANCZOS2, degree 8: max fit error 1.12e-06
static __constant__ float WPOLY8_K_LANCZOS2[2][9] = {
    {-6.368437609e-02f, 9.247301927e-02f, 4.363743636e-02f, -1.062029447e-01f, 2.455305960e-02f, 1.457026981e-02f, -4.860630306e-03f, -8.406574259e-04f, 3.546052027e-04f},
    {5.731591807e-01f, -6.961574710e-01f, -6.472297458e-02f, 2.239244632e-01f, -1.063087087e-02f, -2.981932153e-02f, 2.372569549e-03f, 2.053395512e-03f, -1.779537914e-04f}};
template <> struct WeightPoly<K_LANCZOS2, 8> {
    static constexpr int HALF = 2;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY8_K_LANCZOS2[j][m]; }
};

// K_LANCZOS3, degree 8: max fit error 4.88e-07
static __constant__ float WPOLY8_K_LANCZOS3[3][9] = {
    {2.431709069e-02f, -3.177962398e-02f, -2.159438587e-02f, 3.811809119e-02f, -4.025457159e-03f, -6.743619638e-03f, 1.409867822e-03f, 4.052975720e-04f, -1.071416215e-04f},
    {-1.350949172e-01f, 9.006240410e-02f, 1.401538636e-01f, -1.034299220e-01f, -4.152389678e-03f, 1.420981639e-02f, -9.953854842e-04f, -8.426428615e-04f, 8.885136568e-05f},
    {6.079271041e-01f, -6.645240963e-01f, -1.122099433e-01f, 1.835606860e-01f, 3.978657976e-03f, -2.018404076e-02f, 3.384757005e-04f, 1.147930225e-03f, -3.430345598e-05f}};
template <> struct WeightPoly<K_LANCZOS3, 8> {
    static constexpr int HALF = 3;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY8_K_LANCZOS3[j][m]; }
};

// K_LANCZOS4, degree 8: max fit error 3.24e-07
static __constant__ float WPOLY8_K_LANCZOS4[4][9] = {
    {-1.266088060e-02f, 1.562042682e-02f, 1.239145835e-02f, -1.897269799e-02f, 7.389239865e-04f, 3.590260956e-03f, -5.133529177e-04f, -2.380817188e-04f, 4.386216033e-05f},
    {5.990948595e-02f, -3.370828630e-02f, -6.744278285e-02f, 4.059144974e-02f, 7.415177655e-03f, -7.345860702e-03f, 1.534183975e-04f, 4.628797843e-04f, -3.530932229e-05f},
    {-1.664152334e-01f, 8.387349510e-02f, 1.807127884e-01f, -9.569334900e-02f, -1.448763804e-02f, 1.252212683e-02f, 1.694021416e-04f, -7.025411724e-04f, 2.068797774e-05f},
    {6.203830139e-01f, -6.526052374e-01f, -1.283732447e-01f, 1.686102986e-01f, 8.130628343e-03f, -1.687146911e-02f, -1.339791538e-04f, 8.667293713e-04f, -6.420909172e-06f}};
template <> struct WeightPoly<K_LANCZOS4, 8> {
    static constexpr int HALF = 4;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY8_K_LANCZOS4[j][m]; }
};

// K_REF6, degree 6: max fit error 7.86e-05
static __constant__ float WPOLY6_K_REF6[3][7] = {
    {-2.292518861e-02f, -8.863558629e-03f, 3.976407031e-02f, 8.751609571e-03f, -1.965697040e-02f, 1.237797054e-04f, 2.822262224e-03f},
    {-6.368630864e-02f, 9.240433142e-02f, 4.370697350e-02f, -1.055850624e-01f, 2.417079599e-02f, 1.321160688e-02f, -4.198370374e-03f},
    {5.731601505e-01f, -6.959896936e-01f, -6.475787085e-02f, 2.224152197e-01f, -1.043903708e-02f, -2.650064226e-02f, 2.040223422e-03f}};
template <> struct WeightPoly<K_REF6, 6> {
    static constexpr int HALF = 3;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY6_K_REF6[j][m]; }
};

// K_LANCZOS2, degree 6: max fit error 7.86e-05
static __constant__ float WPOLY6_K_LANCZOS2[2][7] = {
    {-6.368630864e-02f, 9.240433142e-02f, 4.370697350e-02f, -1.055850624e-01f, 2.417079599e-02f, 1.321160688e-02f, -4.198370374e-03f},
    {5.731601505e-01f, -6.959896936e-01f, -6.475787085e-02f, 2.224152197e-01f, -1.043903708e-02f, -2.650064226e-02f, 2.040223422e-03f}};
template <> struct WeightPoly<K_LANCZOS2, 6> {
    static constexpr int HALF = 2;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY6_K_LANCZOS2[j][m]; }
};

// K_LANCZOS3, degree 6: max fit error 4.28e-05
static __constant__ float WPOLY6_K_LANCZOS3[3][7] = {
    {2.431767460e-02f, -3.174650821e-02f, -2.161539606e-02f, 3.782019792e-02f, -3.909958731e-03f, -6.088581365e-03f, 1.209770354e-03f},
    {-1.350954015e-01f, 8.999355403e-02f, 1.401712872e-01f, -1.028105804e-01f, -4.248171251e-03f, 1.284794462e-02f, -8.294468602e-04f},
    {6.079272911e-01f, -6.644303020e-01f, -1.122166701e-01f, 1.827169586e-01f, 4.015637025e-03f, -1.832876631e-02f, 2.744106381e-04f}};
template <> struct WeightPoly<K_LANCZOS3, 6> {
    static constexpr int HALF = 3;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY6_K_LANCZOS3[j][m]; }
};

// K_LANCZOS4, degree 6: max fit error 3.20e-05
static __constant__ float WPOLY6_K_LANCZOS4[4][7] = {
    {-1.266111964e-02f, 1.560097381e-02f, 1.240005960e-02f, -1.879770819e-02f, 6.916406761e-04f, 3.205475434e-03f, -4.314360391e-04f},
    {5.990967838e-02f, -3.367046564e-02f, -6.744970692e-02f, 4.025123361e-02f, 7.453241026e-03f, -6.597758579e-03f, 8.747478137e-05f},
    {-1.664153461e-01f, 8.381609236e-02f, 1.807168453e-01f, -9.517698201e-02f, -1.450993963e-02f, 1.138668614e-02f, 2.080389654e-04f},
    {6.203830489e-01f, -6.525344193e-01f, -1.283745038e-01f, 1.679732535e-01f, 8.137550069e-03f, -1.547066894e-02f, -1.459708303e-04f}};
template <> struct WeightPoly<K_LANCZOS4, 6> {
    static constexpr int HALF = 4;
    static __device__ __forceinline__ float c(int j, int m) { return WPOLY6_K_LANCZOS4[j][m]; }
};

}  // namespace rcabf
