// Compile-time-sized shared-memory FFT of one row by a whole CTA (NT threads), written for
// this project. With M a template constant every index is a shift or a mask and the pass
// schedule unrolls.
#pragma once
#include <vector>

#include "fft.cuh"

namespace nse2d {

template <int X> struct ilog2 { static constexpr int v = 1 + ilog2<X / 2>::v; };
template <> struct ilog2<1> { static constexpr int v = 0; };

// twiddle load through the read-only path
__device__ __forceinline__ cpx<double> ldtw(const cpx<double>* tw, int i) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(tw) + i);
    return {v.x, v.y};
}
__device__ __forceinline__ cpx<float> ldtw(const cpx<float>* tw, int i) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(tw) + i);
    return {v.x, v.y};
}

// Number of passes of an M-point transform: radix 8 while 8 divides what is left, then 4 or 2.
template <int M> struct fft_npass {
    template <int NS> static constexpr int count() {
        if constexpr (NS >= M) return 0;
        else {
            constexpr int REM = M / NS;
            constexpr int R = (REM % 8 == 0) ? 8 : REM;
            return 1 + count<NS * R>();
        }
    }
    static constexpr int v = count<1>();
};

// ---------------------------------------------------------------------------------------
// In-place decimation-in-time FFT of M points in ONE shared buffer.
//
// Pass p (radix R_p, sub-transform length L' = R_0 ... R_{p-1} before it, L = R_p L'):
//   for every group g (start g L) and m in [0, L'):  x_r = buf[g L + m + r L'] * W_L^{r m},
//   y = DFT_R(x), buf[g L + m + s L'] = y_s.
// The input must sit in mixed-radix digit-reversed order: element n of the sequence goes to
// position dit_pos(n); the output is then in natural order. With the radix list
// (R_0, .., R_{P-1}) written most-significant-last, position p = sum d_q (R_0..R_{q-1})
// holds element n = d_{P-1} + R_{P-1} (d_{P-2} + R_{P-2} (...)). Radices: 8 while 8 divides
// what is left, then one 4 or 2.
//
// Shared-memory layout: ip_idx(i) = i + i/8 + i/512 (16-byte units) spreads the stride-8 and
// stride-512 accesses of the first pass and of the digit-reversed scatter over the banks.
//
// Twiddles: a pass with sub-transform length LP > 1 (always a power of 8) reads the pairs
// (W_L^m, W_L^{4m}), L = R LP, m < LP, from a per-pass table, contiguous in m and stored as
// consecutive complex pairs from pair (LP - 8) / 7 on (pass_twiddle_table builds it), so a
// warp's twiddle loads cover consecutive addresses.
// ---------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ int ip_idx(int i) { return i + (i >> 3) + (i >> 9); }
__host__ __device__ constexpr int ip_size(int M) { return M + (M >> 3) + (M >> 9) + 1; }

// Radices are powers of two, so digits are bit groups: pass q has 3 bits (radix 8) except a
// last pass of 1 or 2 bits. Digit d_q sits at bit offset 3q of the position p and is taken from
// n starting at its least significant end in the order q = P-1, P-2, ..., 0.
template <int M> struct ip_plan {
    static constexpr int m = ilog2<M>::v;
    static constexpr int P = fft_npass<M>::v;
    static constexpr int bits(int q) { return (q < m / 3) ? 3 : m % 3; }
};

template <int M> __host__ __device__ __forceinline__ int dit_pos(int n) {
    constexpr int P = ip_plan<M>::P;
    int p = 0, sn = 0;
#pragma unroll
    for (int q = P - 1; q >= 0; --q) {
        const int b = ip_plan<M>::bits(q);
        p |= ((n >> sn) & ((1 << b) - 1)) << (3 * q);
        sn += b;
    }
    return p;
}

// Per-pass twiddle table of an M-point transform from the full table tw[t] = W_M^t: for each
// pass with LP > 1, the pairs (W_L^m, W_L^{4m}) = (tw[m M/L], tw[4 m M/L mod M]), m < LP.
template <typename C>
inline void pass_twiddle_table(int M, const C* tw, std::vector<C>& out) {
    out.clear();
    for (int LP = 8; LP < M; LP *= 8) {
        const int rem = M / LP, R = (rem % 8 == 0) ? 8 : rem, L = R * LP, step = M / L;
        for (int m = 0; m < LP; ++m) {
            out.push_back(tw[(step * m) & (M - 1)]);
            out.push_back(tw[(4 * step * m) & (M - 1)]);
        }
    }
    if (out.empty()) out.push_back(tw[0]);
}

template <typename T, int M, int R, int LP, bool INV, int NT>
__device__ __forceinline__ void ip_pass(cpx<T>* __restrict__ buf, const cpx<T>* __restrict__ tw) {
    constexpr int NB = M / R;            // butterflies
#pragma unroll
    for (int b0 = 0; b0 < NB; b0 += NT) {
        const int b = b0 + (int)threadIdx.x;
        if (NB % NT != 0 && b >= NB) break;
        const int m = b & (LP - 1);
        const int base = (b - m) * R + m;            // g L + m with g = b / LP
        cpx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = buf[ip_idx(base + r * LP)];
        if (LP > 1 && m > 0) {
            // this pass's pair (W_L^m, W_L^{4m}) sits at 2 (off + m) of the per-pass table
            static_assert(LP == 1 || (ilog2<LP>::v % 3 == 0), "passes with twiddles start at a power of 8");
            constexpr int OFF = (LP - 8) / 7;
            cpx<T> wp[R];
            wp[1] = ldtw(tw, 2 * (OFF + m));
            if constexpr (R >= 4) {
                wp[2] = cmul(wp[1], wp[1]);
                wp[3] = cmul(wp[2], wp[1]);
            }
            if constexpr (R == 8) {
                wp[4] = ldtw(tw, 2 * (OFF + m) + 1);
                wp[5] = cmul(wp[4], wp[1]);
                wp[6] = cmul(wp[4], wp[2]);
                wp[7] = cmul(wp[4], wp[3]);
            }
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = INV ? cmulc(v[r], wp[r]) : cmul(v[r], wp[r]);
        }
        dftR<T, R, INV>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) buf[ip_idx(base + r * LP)] = v[r];
    }
}

template <typename T, int M, int LP, bool INV, int NT>
__device__ __forceinline__ void ip_passes(cpx<T>* buf, const cpx<T>* tw) {
    if constexpr (LP < M) {
        constexpr int REM = M / LP;
        constexpr int R = (REM % 8 == 0) ? 8 : REM;
        ip_pass<T, M, R, LP, INV, NT>(buf, tw);
        __syncthreads();
        ip_passes<T, M, LP * R, INV, NT>(buf, tw);
    }
}

// ---------------------------------------------------------------------------------------
// Radix-16 plan of the FP64 row transforms: passes of radix 16, the last one of the remaining
// 1..4 bits. Pass 0 reads its 16 points straight from global memory into registers: with the
// digit-reversed layout, the butterfly that starts at position dit16_pos(t) (t < M/16) holds
// the points t + (M/16) r, r < 16, so thread t loads a coalesced column of the row and writes
// its 16 outputs to positions dit16_pos(t) + s. Later passes exchange through shared memory as
// above (same padding). Twiddles of pass q >= 1 come from a table of (W^m, W^2m, W^4m, W^8m),
// L = R LP, m < LP; W^(r m) is applied as W^(a m) W^(4 b m) with r = a + 4 b, so that at most
// six twiddles are live at a time.
// ---------------------------------------------------------------------------------------
template <int M> struct p16_plan {
    static constexpr int m = ilog2<M>::v;
    static constexpr int P = (m + 3) / 4;
    static constexpr int bits(int q) { return (q < P - 1) ? 4 : m - 4 * (P - 1); }
    static constexpr int R(int q) { return 1 << bits(q); }
    static constexpr int LP(int q) { return 1 << (4 * q); }
    static constexpr int off(int q) {           // first table entry of pass q >= 1
        int o = 0;
        for (int i = 1; i < q; ++i) o += 4 * LP(i);
        return o;
    }
};

template <int M> __host__ __device__ __forceinline__ int dit16_pos(int n) {
    constexpr int P = p16_plan<M>::P;
    int p = 0, sn = 0;
#pragma unroll
    for (int q = P - 1; q >= 0; --q) {
        const int b = p16_plan<M>::bits(q);
        p |= ((n >> sn) & ((1 << b) - 1)) << (4 * q);
        sn += b;
    }
    return p;
}

template <typename C>
inline void p16_twiddle_table(int M, const C* tw, std::vector<C>& out) {
    out.clear();
    int m = 0;
    while ((1 << m) < M) ++m;
    const int P = (m + 3) / 4;
    for (int q = 1; q < P; ++q) {
        const int LP = 1 << (4 * q), R = 1 << ((q < P - 1) ? 4 : m - 4 * (P - 1)), L = R * LP, step = M / L;
        for (int k = 0; k < LP; ++k)
            for (int e = 1; e <= 8; e *= 2) out.push_back(tw[((long long)e * step * k) % M]);
    }
    if (out.empty()) out.push_back(tw[0]);
}

template <typename T, bool INV> __device__ __forceinline__ cpx<T> p16_tw(cpx<T> a, cpx<T> w) {
    return INV ? cmulc(a, w) : cmul(a, w);
}

template <typename T, int M, int Q, bool INV, int NT>
__device__ __forceinline__ void p16_pass(cpx<T>* __restrict__ buf, const cpx<T>* __restrict__ tw) {
    constexpr int R = p16_plan<M>::R(Q), LP = p16_plan<M>::LP(Q), NB = M / R, OFF = p16_plan<M>::off(Q);
#pragma unroll 1
    for (int b0 = 0; b0 < NB; b0 += NT) {
        const int b = b0 + (int)threadIdx.x;
        if (NB % NT != 0 && b >= NB) break;
        const int mm = b & (LP - 1);
        const int base = (b - mm) * R + mm;
        cpx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = buf[ip_idx(base + r * LP)];
        if (mm > 0) {
            const int t = OFF + 4 * mm;
            const cpx<T> w1 = ldtw(tw, t);
            if constexpr (R == 2) {
                v[1] = p16_tw<T, INV>(v[1], w1);
            } else {
                const cpx<T> w2 = ldtw(tw, t + 1), w3 = cmul(w1, w2);
#pragma unroll
                for (int r = 1; r < R; ++r) {                  // low digit a = r mod 4
                    const int a = r & 3;
                    if (a) v[r] = p16_tw<T, INV>(v[r], a == 1 ? w1 : (a == 2 ? w2 : w3));
                }
                if constexpr (R >= 8) {                        // high digit b = r / 4
                    const cpx<T> w4 = ldtw(tw, t + 2);
                    cpx<T> w8 = w4, w12 = w4;
                    if constexpr (R == 16) {
                        w8 = ldtw(tw, t + 3);
                        w12 = cmul(w4, w8);
                    }
#pragma unroll
                    for (int r = 4; r < R; ++r) {
                        const int hb = r >> 2;
                        v[r] = p16_tw<T, INV>(v[r], hb == 1 ? w4 : (hb == 2 ? w8 : w12));
                    }
                }
            }
        }
        dftR<T, R, INV>(v);
#pragma unroll
        for (int r = 0; r < R; ++r) buf[ip_idx(base + r * LP)] = v[r];
    }
}

template <typename T, int M, int Q, bool INV, int NT>
__device__ __forceinline__ void p16_passes_from(cpx<T>* buf, const cpx<T>* tw) {
    if constexpr (Q < p16_plan<M>::P) {
        p16_pass<T, M, Q, INV, NT>(buf, tw);
        __syncthreads();
        p16_passes_from<T, M, Q + 1, INV, NT>(buf, tw);
    }
}

}  // namespace nse2d
