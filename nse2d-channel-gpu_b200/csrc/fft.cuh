// Complex arithmetic and the in-register 2/4/8-point DFTs of the row FFTs (FP64 or FP32),
// written for this project.
//
// The reference transforms real rows with cuFFT Z2Z (src/poisson.cuh:36-37,96,110): a
// complex transform of length Nx on data whose imaginary part is zero. Here a row of
// Nx reals is transformed as Nx/2 complex points z_n = x_{2n} + i x_{2n+1} (the row in
// memory, reinterpreted), followed by the split step that separates the even and odd
// samples. Only the half spectrum k = 0..Nx/2 is produced and consumed, which is all a
// real field needs. The passes themselves live in fft_rows.cuh.
//
// Every function here is __host__ __device__, so the same butterflies can be stepped on the
// CPU to check index arithmetic and numerics before they run on a GPU.
#pragma once

#ifdef __CUDACC__
#define NSE_HD __host__ __device__ __forceinline__
#else
#define NSE_HD inline
#endif

namespace nse2d {

// Aligned to its full size, so that a complex element moves as one 16-byte (FP64) or 8-byte
// (FP32) access to shared or global memory.
template <typename T> struct alignas(2 * sizeof(T)) cpx { T x, y; };

template <typename T> NSE_HD cpx<T> cmul(cpx<T> a, cpx<T> b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <typename T> NSE_HD cpx<T> cmulc(cpx<T> a, cpx<T> b) { return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y}; }  // a * conj(b)
template <typename T> NSE_HD cpx<T> cadd(cpx<T> a, cpx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T> NSE_HD cpx<T> csub(cpx<T> a, cpx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T> NSE_HD cpx<T> mul_mi(cpx<T> a) { return {a.y, -a.x}; }   // a * (-i)
template <typename T> NSE_HD cpx<T> mul_pi(cpx<T> a) { return {-a.y, a.x}; }   // a * (+i)

// In-register DFT of 2, 4 or 8 points, forward (e^{-i}) when INV is false.
template <typename T, bool INV> NSE_HD void dft2(cpx<T>* v) {
    cpx<T> a = v[0], b = v[1];
    v[0] = cadd(a, b); v[1] = csub(a, b);
}
template <typename T, bool INV> NSE_HD void dft4(cpx<T>* v) {
    cpx<T> a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
    cpx<T> b0 = cadd(v[1], v[3]), b1 = csub(v[1], v[3]);
    b1 = INV ? mul_pi(b1) : mul_mi(b1);
    v[0] = cadd(a0, b0); v[2] = csub(a0, b0);
    v[1] = cadd(a1, b1); v[3] = csub(a1, b1);
}
template <typename T, bool INV> NSE_HD void dft8(cpx<T>* v) {
    // radix-2 split into even/odd 4-point DFTs, then combine with e^{-/+ 2 pi i k/8}
    const T s = (T)0.70710678118654752440084436210484903928;   // 1/sqrt(2)
    cpx<T> e[4] = {v[0], v[2], v[4], v[6]};
    cpx<T> o[4] = {v[1], v[3], v[5], v[7]};
    dft4<T, INV>(e); dft4<T, INV>(o);
    // o_k *= w^k, w = e^{-i pi/4} (forward) or e^{+i pi/4} (inverse)
    cpx<T> o1 = INV ? cpx<T>{(o[1].x - o[1].y) * s, (o[1].x + o[1].y) * s}
                    : cpx<T>{(o[1].x + o[1].y) * s, (o[1].y - o[1].x) * s};
    cpx<T> o2 = INV ? mul_pi(o[2]) : mul_mi(o[2]);
    cpx<T> o3 = INV ? cpx<T>{-(o[3].x + o[3].y) * s, (o[3].x - o[3].y) * s}
                    : cpx<T>{(o[3].y - o[3].x) * s, -(o[3].x + o[3].y) * s};
    v[0] = cadd(e[0], o[0]); v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);   v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);   v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);   v[7] = csub(e[3], o3);
}

// 16-point DFT as 4 x 4: four 4-point DFTs over x[4 n1 + n2] (n1), the twiddles W16^(n2 k1),
// four 4-point DFTs over n2; X[k1 + 4 k2]. W16^j = e^{-/+ 2 pi i j / 16}: cos(pi/8), sin(pi/8)
// and 1/sqrt(2) are the only constants.
template <typename T> NSE_HD cpx<T> mul_w16(cpx<T> a, int j, bool inv) {
    const T c = (T)0.92387953251128675612818318939678828682;   // cos(pi/8)
    const T s = (T)0.38268343236508977172845998403039886676;   // sin(pi/8)
    const T r = (T)0.70710678118654752440084436210484903928;   // 1/sqrt(2)
    // forward W16^j = (cos(2 pi j/16), -sin(2 pi j/16)); inverse conjugated
    T wr, wi;
    switch (j) {
        case 1: wr = c; wi = -s; break;
        case 2: wr = r; wi = -r; break;
        case 3: wr = s; wi = -c; break;
        case 6: wr = -r; wi = -r; break;
        case 9: wr = -c; wi = s; break;
        default: wr = 1; wi = 0; break;                          // j = 0 (j = 4 is handled by the caller)
    }
    if (inv) wi = -wi;
    return {a.x * wr - a.y * wi, a.x * wi + a.y * wr};
}
// e^{-i pi r / 16}, r = 0..15, from cos and sin of pi/16, pi/8, 3 pi/16, pi/4 (the doubles
// nearest the exact values): the factor W_{2M}^{(M/16) r} that relates the split/merge twiddles
// W_{2M}^n of the points n = t + (M/16) r to W_{2M}^t, whatever M.
template <typename T> NSE_HD cpx<T> w32(int r) {
    const T c1 = (T)0.98078528040323044912618223613424, s1 = (T)0.19509032201612826784828486847702;
    const T c2 = (T)0.92387953251128675612818318939679, s2 = (T)0.38268343236508977172845998403040;
    const T c3 = (T)0.83146961230254523707878837761791, s3 = (T)0.55557023301960222474283081394853;
    const T h = (T)0.70710678118654752440084436210485;
    switch (r & 15) {
        case 0: return {(T)1, (T)0};   case 1: return {c1, -s1};   case 2: return {c2, -s2};
        case 3: return {c3, -s3};      case 4: return {h, -h};     case 5: return {s3, -c3};
        case 6: return {s2, -c2};      case 7: return {s1, -c1};   case 8: return {(T)0, (T)-1};
        case 9: return {-s1, -c1};     case 10: return {-s2, -c2}; case 11: return {-s3, -c3};
        case 12: return {-h, -h};      case 13: return {-c3, -s3}; case 14: return {-c2, -s2};
        default: return {-c1, -s1};
    }
}

template <typename T, bool INV> NSE_HD void dft16(cpx<T>* v) {
    cpx<T> y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
        cpx<T> q[4] = {v[n2], v[4 + n2], v[8 + n2], v[12 + n2]};
        dft4<T, INV>(q);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            const int j = n2 * k1;
            if (j == 0) y[n2][k1] = q[k1];
            else if (j == 4) y[n2][k1] = INV ? mul_pi(q[k1]) : mul_mi(q[k1]);
            else y[n2][k1] = mul_w16(q[k1], j, INV);
        }
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
        cpx<T> q[4] = {y[0][k1], y[1][k1], y[2][k1], y[3][k1]};
        dft4<T, INV>(q);
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = q[k2];
    }
}

template <typename T, int R, bool INV> NSE_HD void dftR(cpx<T>* v) {
    if constexpr (R == 2) dft2<T, INV>(v);
    else if constexpr (R == 4) dft4<T, INV>(v);
    else if constexpr (R == 8) dft8<T, INV>(v);
    else dft16<T, INV>(v);
}

}  // namespace nse2d
