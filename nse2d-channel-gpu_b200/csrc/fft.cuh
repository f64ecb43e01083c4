// Shared-memory real FFT along x for one row (FP64 or FP32), written for this project.
//
// The reference transforms real rows with cuFFT Z2Z (src/poisson.cuh:36-37,96,110): a
// complex transform of length Nx on data whose imaginary part is zero. Here a row of
// Nx reals is transformed as Nx/2 complex points z_n = x_{2n} + i x_{2n+1} (the row in
// memory, reinterpreted), followed by the split step that separates the even and odd
// samples. Only the half spectrum k = 0..Nx/2 is produced and consumed, which is all a
// real field needs.
//
// The complex transform is a Stockham auto-sort FFT (no bit reversal) with radix-8,
// radix-4 and radix-2 passes. Pass p reads buffer A and writes buffer B:
//   for butterfly j in [0, M/R):  v_r = A[j + r M/R] * w^(r (j mod Ns)),  w = e^{-2 pi i/(Ns R)}
//                                 V = DFT_R(v);  B[(j/Ns) Ns R + (j mod Ns) + r Ns] = V_r
// with Ns the product of the radices of the earlier passes. Twiddles come from a table
// tw[t] = e^{-2 pi i t / M} (t < M) computed on the host in long double.
//
// Every function here is __host__ __device__ and takes the thread index explicitly, so
// the same code can be stepped on the CPU (one "thread" at a time, a pass at a time)
// to check the index arithmetic against numpy before it runs on a GPU.
#pragma once

#ifdef __CUDACC__
#define NSE_HD __host__ __device__ __forceinline__
#else
#define NSE_HD inline
#endif

namespace nse2d {

template <typename T> struct cpx { T x, y; };

template <typename T> NSE_HD cpx<T> cmul(cpx<T> a, cpx<T> b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <typename T> NSE_HD cpx<T> cmulc(cpx<T> a, cpx<T> b) { return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y}; }  // a * conj(b)
template <typename T> NSE_HD cpx<T> cadd(cpx<T> a, cpx<T> b) { return {a.x + b.x, a.y + b.y}; }
template <typename T> NSE_HD cpx<T> csub(cpx<T> a, cpx<T> b) { return {a.x - b.x, a.y - b.y}; }
template <typename T> NSE_HD cpx<T> mul_mi(cpx<T> a) { return {a.y, -a.x}; }   // a * (-i)
template <typename T> NSE_HD cpx<T> mul_pi(cpx<T> a) { return {-a.y, a.x}; }   // a * (+i)

// Shared-memory index with one pad element every 8 (breaks the stride-R bank conflicts of
// the first passes). A buffer of M elements occupies padded_size(M) slots.
NSE_HD int pad_idx(int i) { return i + (i >> 3); }
NSE_HD int padded_size(int M) { return M + (M >> 3) + 1; }

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

template <typename T, int R, bool INV> NSE_HD void dftR(cpx<T>* v) {
    if constexpr (R == 2) dft2<T, INV>(v);
    else if constexpr (R == 4) dft4<T, INV>(v);
    else dft8<T, INV>(v);
}

// One butterfly j of a radix-R Stockham pass on M points (see the header comment).
// tw: table of M twiddles e^{-2 pi i t/M}. in/out: padded shared-memory buffers.
template <typename T, int R, bool INV>
NSE_HD void stockham_butterfly(int j, int M, int Ns, const cpx<T>* __restrict__ in,
                               cpx<T>* __restrict__ out, const cpx<T>* __restrict__ tw) {
    const int stride = M / R;
    const int k = j % Ns;                 // position inside the current sub-transform
    const int tstep = (M / (Ns * R)) * k; // twiddle index step for r = 1
    cpx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        cpx<T> a = in[pad_idx(j + r * stride)];
        if (r > 0 && k > 0) {
            const cpx<T> w = tw[(r * tstep) & (M - 1)];
            a = INV ? cmulc(a, w) : cmul(a, w);
        }
        v[r] = a;
    }
    dftR<T, R, INV>(v);
    const int base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) out[pad_idx(base + r * Ns)] = v[r];
}

// The pass schedule for M = 2^m points: radix-8 passes, then one radix-4 or radix-2.
// Returns the number of passes and fills radix[].
NSE_HD int fft_schedule(int M, int* radix) {
    int n = 0, rem = M;
    while (rem >= 8 && (rem % 8) == 0) { radix[n++] = 8; rem /= 8; }
    if (rem == 4) radix[n++] = 4;
    else if (rem == 2) radix[n++] = 2;
    return n;
}

// Split step of the forward real transform: Z (M points, FFT of z_n = x_2n + i x_2n+1)
// to X_k, k = k (one value; 0 <= k <= M), N = 2M:
//   E_k = (Z_k + conj Z_{M-k}) / 2,  O_k = -i (Z_k - conj Z_{M-k}) / 2,  X_k = E_k + W_N^k O_k
// with Z_M = Z_0 and W_N^k = e^{-2 pi i k/N} from the table wN (M + 1 entries).
template <typename T>
NSE_HD cpx<T> rfft_split(int k, int M, const cpx<T>* __restrict__ Z, const cpx<T>* __restrict__ wN) {
    const cpx<T> a = Z[pad_idx(k == M ? 0 : k)];
    const cpx<T> b0 = Z[pad_idx(k == 0 ? 0 : M - k)];
    const cpx<T> b = {b0.x, -b0.y};                  // conj Z_{M-k}
    const cpx<T> E = {(T)0.5 * (a.x + b.x), (T)0.5 * (a.y + b.y)};
    const cpx<T> D = {(T)0.5 * (a.x - b.x), (T)0.5 * (a.y - b.y)};
    const cpx<T> O = mul_mi(D);
    return cadd(E, cmul(wN[k], O));
}

// Merge step of the inverse real transform: half spectrum X_k (k = 0..M) to the M-point
// complex sequence Z_k whose inverse FFT gives z_n = x_2n + i x_2n+1 (times M; the caller
// scales by 1/N overall to get the inverse DFT of the full Hermitian spectrum, times 2):
//   E_k = (X_k + conj X_{M-k}) / 2,  O_k = (X_k - conj X_{M-k}) W_N^{-k} / 2,  Z_k = E_k + i O_k
template <typename T>
NSE_HD cpx<T> irfft_merge(int k, int M, const cpx<T>* __restrict__ X, const cpx<T>* __restrict__ wN) {
    const cpx<T> a = X[k];
    const cpx<T> b0 = X[M - k];
    const cpx<T> b = {b0.x, -b0.y};
    const cpx<T> E = {(T)0.5 * (a.x + b.x), (T)0.5 * (a.y + b.y)};
    const cpx<T> D = {(T)0.5 * (a.x - b.x), (T)0.5 * (a.y - b.y)};
    const cpx<T> O = cmulc(D, wN[k]);               // D * conj(W_N^k) = D * W_N^{-k}
    return cadd(E, mul_pi(O));
}

}  // namespace nse2d
