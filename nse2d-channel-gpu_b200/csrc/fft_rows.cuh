// Compile-time-sized shared-memory FFT of one row by a whole CTA (NT threads).
// Written for this project; the pass formula is the Stockham auto-sort form documented in
// fft.cuh. With M a template constant every index is a shift or a mask, the pass schedule
// unrolls, and the first pass reads an unpadded buffer (its stride-M/R reads are already
// conflict free), so a row can be staged into that buffer with plain vector loads.
//
// Buffers: A = M elements unpadded, B = padded_size(M) elements. Pass p reads the buffer
// written by pass p-1 (A for p = 0) and writes B when p is even, A when p is odd. Only the
// first pass (sub-transform length 1, stride-R stores) needs the padded layout; later
// passes store runs of at least 8 consecutive elements per 8 lanes.
#pragma once
#include "fft.cuh"

namespace nse2d {

template <int X> struct ilog2 { static constexpr int v = 1 + ilog2<X / 2>::v; };
template <> struct ilog2<1> { static constexpr int v = 0; };

template <bool PAD> __device__ __forceinline__ int bidx(int i) { return PAD ? pad_idx(i) : i; }

// twiddle load through the read-only path
__device__ __forceinline__ cpx<double> ldtw(const cpx<double>* tw, int i) {
    const double2 v = __ldg(reinterpret_cast<const double2*>(tw) + i);
    return {v.x, v.y};
}
__device__ __forceinline__ cpx<float> ldtw(const cpx<float>* tw, int i) {
    const float2 v = __ldg(reinterpret_cast<const float2*>(tw) + i);
    return {v.x, v.y};
}

template <typename T, int M, int R, int NS, bool INV, bool IN_PAD, bool OUT_PAD, int NT>
__device__ __forceinline__ void fft_pass(const cpx<T>* __restrict__ in, cpx<T>* __restrict__ out,
                                         const cpx<T>* __restrict__ tw) {
    constexpr int NB = M / R;
    constexpr int STRIDE = M / R;
    constexpr int TSTEP = M / (NS * R);
#pragma unroll
    for (int j0 = 0; j0 < NB; j0 += NT) {
        const int j = j0 + (int)threadIdx.x;
        if (NB % NT != 0 && j >= NB) break;
        const int k = j & (NS - 1);
        cpx<T> v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = in[bidx<IN_PAD>(j + r * STRIDE)];
        if (NS > 1 && k > 0) {
            // w^r for r = 1..R-1 from two table loads (w and w^4 for radix 8): a few complex
            // products instead of R-1 dependent loads
            cpx<T> wp[R];
            wp[1] = ldtw(tw, (TSTEP * k) & (M - 1));
            if constexpr (R >= 4) {
                wp[2] = cmul(wp[1], wp[1]);
                wp[3] = cmul(wp[2], wp[1]);
            }
            if constexpr (R == 8) {
                wp[4] = ldtw(tw, (4 * TSTEP * k) & (M - 1));
                wp[5] = cmul(wp[4], wp[1]);
                wp[6] = cmul(wp[4], wp[2]);
                wp[7] = cmul(wp[4], wp[3]);
            }
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = INV ? cmulc(v[r], wp[r]) : cmul(v[r], wp[r]);
        }
        dftR<T, R, INV>(v);
        const int base = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) out[bidx<OUT_PAD>(base + r * NS)] = v[r];
    }
}

// All passes: radix-8 while 8 divides the remaining length, then a radix-4 or radix-2 pass.
// Returns (through the template recursion) the parity of the pass count: the result lies in
// B when the number of passes is odd, in A when it is even.
// in0: the unpadded input of pass 0 (may be A itself, or a separate staging buffer that is
// free again once pass 0 is done, so that the next row can be loaded into it meanwhile).
// on_pass0_done() runs right after the barrier that ends pass 0.
template <typename T, int M, int NS, int P, bool INV, int NT, typename F>
__device__ __forceinline__ void fft_passes(const cpx<T>* in0, cpx<T>* A, cpx<T>* B, const cpx<T>* tw,
                                           F&& on_pass0_done) {
    if constexpr (NS < M) {
        constexpr int REM = M / NS;
        constexpr int R = (REM % 8 == 0) ? 8 : REM;   // REM is 4 or 2 in the last pass
        constexpr bool IN_PAD = (P % 2 == 1);         // pass P reads what pass P-1 wrote
        constexpr bool OUT_PAD = (P % 2 == 0);
        const cpx<T>* in = (P == 0) ? in0 : ((P % 2 == 0) ? A : B);
        cpx<T>* out = (P % 2 == 0) ? B : A;
        fft_pass<T, M, R, NS, INV, IN_PAD, OUT_PAD, NT>(in, out, tw);
        __syncthreads();
        if constexpr (P == 0) on_pass0_done();
        fft_passes<T, M, NS * R, P + 1, INV, NT>(in0, A, B, tw, on_pass0_done);
    }
}

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

// Result buffer of an M-point transform run by fft_passes: B (padded) if the pass count is odd.
template <int M> struct fft_out { static constexpr bool in_B = (fft_npass<M>::v % 2) == 1; };

}  // namespace nse2d
