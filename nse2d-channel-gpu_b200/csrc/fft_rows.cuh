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

// Shared-memory layout of a row of M points: ip_idx<M>(i) = i + (i >> A) + (i >> B) (in elements)
// spreads the digit-reversed writes of the first pass, the strided accesses of the later passes
// and the split step's descending reads over the banks. A and B are chosen per M by counting
// the shared-memory wavefronts of all of these accesses, for 16-byte (FP64) and 8-byte (FP32)
// elements; at M = 2048 every access is conflict-free (one pad element per 256).
__host__ __device__ constexpr int ip_shift_a(int M) { return M >= 8192 ? 7 : (M >= 2048 ? 8 : 4); }
__host__ __device__ constexpr int ip_shift_b(int M) {
    return M == 64 ? 6 : M == 128 ? 7 : M == 256 ? 8 : M == 512 ? 6 : M == 1024 ? 7 : M == 2048 ? 11 : M >= 4096 ? 12 : 30;
}
template <int M> __host__ __device__ __forceinline__ int ip_idx(int i) {
    return i + (i >> ip_shift_a(M)) + (i >> ip_shift_b(M));
}
__host__ __device__ constexpr int ip_size(int M) {
    return M + ((M - 1) >> ip_shift_a(M)) + ((M - 1) >> ip_shift_b(M));
}

// ---------------------------------------------------------------------------------------
// Radix-16 plan of the row transforms (FP64 and FP32): in-place decimation-in-time passes of
// radix 16, the last one of the remaining 1..4 bits.
//
// Pass 0 reads its 16 points straight from global memory into registers: with the
// digit-reversed layout, the butterfly that starts at position dit16_pos(t) (t < M/16) holds
// the points t + (M/16) r, r < 16, so thread t loads a coalesced column of the row and writes
// its 16 outputs to positions dit16_pos(t) + s.
//
// Pass q >= 1 (radix R, sub-transform length LP = 16^q before it, L = R LP), for every group g
// and m < LP: x_r = buf[g L + m + r LP] times W_L^(r m), an R-point DFT, written back in place.
// The output is in natural order. Its twiddles come from four tables of W^m, W^2m, W^4m and
// W^8m, m < LP (one after the other, so that the lanes of a warp, which take consecutive m,
// read consecutive entries); W^(r m) is applied as W^(a m) W^(4 b m) with r = a + 4 b, so that
// at most six twiddles are live at a time.
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
        for (int e = 1; e <= 8; e *= 2)
            for (int k = 0; k < LP; ++k) out.push_back(tw[((long long)e * step * k) % M]);
    }
    if (out.empty()) out.push_back(tw[0]);
}

template <typename T, bool INV> __device__ __forceinline__ cpx<T> p16_tw(cpx<T> a, cpx<T> w) {
    return INV ? cmulc(a, w) : cmul(a, w);
}

// One pass q >= 1 of the plan over the buffer; its outputs go to out(position, value), by
// default back into the buffer.
template <typename T, int M, int Q, bool INV, int NT, typename Out>
__device__ __forceinline__ void p16_pass_to(cpx<T>* __restrict__ buf, const cpx<T>* __restrict__ tw, Out out);

template <typename T, int M, int Q, bool INV, int NT>
__device__ __forceinline__ void p16_pass(cpx<T>* __restrict__ buf, const cpx<T>* __restrict__ tw) {
    p16_pass_to<T, M, Q, INV, NT>(buf, tw, [&](int pos, const cpx<T>& v) { buf[ip_idx<M>(pos)] = v; });
}

// Butterfly b of pass q >= 1: loads its R points from the buffer, applies the twiddles and the
// R-point DFT; v[r] is then the output at position base + r LP (returned in base).
template <typename T, int M, int Q, bool INV>
__device__ __forceinline__ int p16_bfly(const cpx<T>* __restrict__ buf, const cpx<T>* __restrict__ tw, int b,
                                        cpx<T> (&v)[p16_plan<M>::R(Q)]) {
    constexpr int R = p16_plan<M>::R(Q), LP = p16_plan<M>::LP(Q), OFF = p16_plan<M>::off(Q);
    const int mm = b & (LP - 1);
    const int base = (b - mm) * R + mm;
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = buf[ip_idx<M>(base + r * LP)];
    if (mm > 0) {
        const int t = OFF + mm;
        const cpx<T> w1 = ldtw(tw, t);
        if constexpr (R == 2) {
            v[1] = p16_tw<T, INV>(v[1], w1);
        } else {
            const cpx<T> w2 = ldtw(tw, t + LP), w3 = cmul(w1, w2);
#pragma unroll
            for (int r = 1; r < R; ++r) {                  // low digit a = r mod 4
                const int a = r & 3;
                if (a) v[r] = p16_tw<T, INV>(v[r], a == 1 ? w1 : (a == 2 ? w2 : w3));
            }
            if constexpr (R >= 8) {                        // high digit b = r / 4
                const cpx<T> w4 = ldtw(tw, t + 2 * LP);
                cpx<T> w8 = w4, w12 = w4;
                if constexpr (R == 16) {
                    w8 = ldtw(tw, t + 3 * LP);
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
    return base;
}

template <typename T, int M, int Q, bool INV, int NT, typename Out>
__device__ __forceinline__ void p16_pass_to(cpx<T>* __restrict__ buf, const cpx<T>* __restrict__ tw, Out out) {
    constexpr int R = p16_plan<M>::R(Q), LP = p16_plan<M>::LP(Q), NB = M / R;
#pragma unroll 1
    for (int b0 = 0; b0 < NB; b0 += NT) {
        const int b = b0 + (int)threadIdx.x;
        if (NB % NT != 0 && b >= NB) break;
        cpx<T> v[R];
        const int base = p16_bfly<T, M, Q, INV>(buf, tw, b, v);
#pragma unroll
        for (int r = 0; r < R; ++r) out(base + r * LP, v[r]);
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

// Passes Q .. P-1 where the last one hands its outputs (natural order) to out(position, value)
// instead of writing them back: the caller stores them to global memory from registers.
// Needs P >= 2 and Q >= 1.
template <typename T, int M, int Q, bool INV, int NT, typename Out>
__device__ __forceinline__ void p16_passes_to(cpx<T>* buf, const cpx<T>* tw, Out out) {
    constexpr int P = p16_plan<M>::P;
    if constexpr (Q < P - 1) {
        p16_pass<T, M, Q, INV, NT>(buf, tw);
        __syncthreads();
        p16_passes_to<T, M, Q + 1, INV, NT>(buf, tw, out);
    } else if constexpr (Q == P - 1) {
        p16_pass_to<T, M, Q, INV, NT>(buf, tw, out);
    }
}

}  // namespace nse2d
