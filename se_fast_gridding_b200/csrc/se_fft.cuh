// se_fft.cuh -- the k-space step (FFT, scaling SE_general.c:145-175, inverse
// FFT) in FP64 for grids of M = 32, 64 or 128, in three passes instead of
// cuFFT's D2Z (three kernels), the scaling pass and Z2D (three kernels).
// Included inside namespace se by se_solve.cu after kwave().
//
//   k_fft_zy       one CTA per x plane: the real z lines in pairs (y, y + M/2)
//                  as one complex line each, unpacked into the two half
//                  spectra, then every kz column along y; the plane's half
//                  spectrum [ky][kz <= M/2] goes out as one block, in cuFFT's
//                  layout [x][ky][kz];
//   k_fft_x_scale  one CTA per (ky, run of kz): each line along x forward,
//                  times Z(k), inverse;
//   k_ifft_yz      one CTA per x plane: every kz column along ky inverse,
//                  then the z lines in pairs from their Hermitian half
//                  spectra, inverse, real parts to row y and imaginary parts
//                  to row y + M/2 of the grid (and of its FP32 copy).
//
// A line of M = N1 N2 points (16 x 8, 8 x 8, 8 x 4) is transformed in place
// in shared memory in two stages: thread n2 < N2 takes the points N2 n1 + n2,
// n1 < N1, through an N1-point DFT in registers and the twiddles
// W_M^(n2 k1), and puts result k1 back in place N2 k1 + n2 (the places it
// read); then thread k1 < N1 takes places N2 k1 + n2, n2 < N2, through an
// N2-point DFT and writes X[k1 + N1 k2] to place k1 + N1 k2: natural order in
// and out, no permutation.  The inverse is the same with conjugate twiddles.
// Unnormalised both ways, as cuFFT and FFTW: the 1/M^3 is in Z.  Twiddles
// W_128^k from a table built on the host in long double; the small DFTs use
// exact constants.

constexpr int FFT_THREADS = 512;

__device__ __forceinline__ double2 c_add(double2 a, double2 b)
{
    return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 c_sub(double2 a, double2 b)
{
    return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 c_mul(double2 a, double2 b)
{
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 c_conj(double2 a) { return make_double2(a.x, -a.y); }
// a times -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ double2 c_rot(double2 a)
{
    return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void dft4(double2& a0, double2& a1, double2& a2, double2& a3)
{
    const double2 s02 = c_add(a0, a2), d02 = c_sub(a0, a2);
    const double2 s13 = c_add(a1, a3), r = c_rot<INV>(c_sub(a1, a3));
    a0 = c_add(s02, s13);
    a2 = c_sub(s02, s13);
    a1 = c_add(d02, r);
    a3 = c_sub(d02, r);
}

// a[k] <- sum_n a[n] W_8^(n k), W_8 = exp(-+ i pi / 4)
template <bool INV>
__device__ __forceinline__ void dft8(double2 (&a)[8])
{
    constexpr double H = 0.70710678118654752440;   // sqrt(1/2)
    double2 e0 = a[0], e1 = a[2], e2 = a[4], e3 = a[6];
    double2 o0 = a[1], o1 = a[3], o2 = a[5], o3 = a[7];
    dft4<INV>(e0, e1, e2, e3);
    dft4<INV>(o0, o1, o2, o3);
    const double sg = INV ? 1.0 : -1.0;
    const double2 w1 = make_double2(H, sg * H), w3 = make_double2(-H, sg * H);
    o1 = c_mul(o1, w1);
    o2 = c_rot<INV>(o2);
    o3 = c_mul(o3, w3);
    a[0] = c_add(e0, o0);
    a[4] = c_sub(e0, o0);
    a[1] = c_add(e1, o1);
    a[5] = c_sub(e1, o1);
    a[2] = c_add(e2, o2);
    a[6] = c_sub(e2, o2);
    a[3] = c_add(e3, o3);
    a[7] = c_sub(e3, o3);
}

// X[k] = sum_n a[n] W_16^(n k), left in a[dig16(k)]: four 4-point DFTs of
// a[4 n1 + n2], the twiddles W_16^(n2 k1), four 4-point DFTs across n2 in
// place (X[k1 + 4 k2] in a[4 k1 + k2]).
__host__ __device__ constexpr int dig16(int k) { return 4 * (k & 3) + (k >> 2); }

template <bool INV>
__device__ __forceinline__ void dft16(double2 (&a)[16])
{
    constexpr double C1 = 0.92387953251128675613, S1 = 0.38268343236508977173;   // 2 pi / 16
    constexpr double H = 0.70710678118654752440;
    const double sg = INV ? 1.0 : -1.0;
#pragma unroll
    for (int n2 = 0; n2 < 4; n2++) dft4<INV>(a[n2], a[4 + n2], a[8 + n2], a[12 + n2]);
    // row k1 (places 4 k1 + n2) times W_16^(n2 k1)
    const double2 w1 = make_double2(C1, sg * S1), w2 = make_double2(H, sg * H),
                  w3 = make_double2(S1, sg * C1), w6 = make_double2(-H, sg * H),
                  w9 = make_double2(-C1, -sg * S1);
    a[5] = c_mul(a[5], w1);
    a[6] = c_mul(a[6], w2);
    a[7] = c_mul(a[7], w3);
    a[9] = c_mul(a[9], w2);
    a[10] = c_rot<INV>(a[10]);
    a[11] = c_mul(a[11], w6);
    a[13] = c_mul(a[13], w3);
    a[14] = c_mul(a[14], w6);
    a[15] = c_mul(a[15], w9);
#pragma unroll
    for (int k1 = 0; k1 < 4; k1++)
        dft4<INV>(a[4 * k1], a[4 * k1 + 1], a[4 * k1 + 2], a[4 * k1 + 3]);
}

// Where an N-point DFT leaves X[k] (N = 16: digit-reversed; 4, 8: in place).
template <int N>
__host__ __device__ constexpr int dft_at(int k) { return N == 16 ? dig16(k) : k; }

// a[dft_at<N>(k)] <- sum_n a[n] W_N^(n k)
template <int N, bool INV>
__device__ __forceinline__ void dft_small(double2 (&a)[N])
{
    if constexpr (N == 4) dft4<INV>(a[0], a[1], a[2], a[3]);
    else if constexpr (N == 8) dft8<INV>(a);
    else dft16<INV>(a);
}

// The line split M = N1 N2.
template <int M>
struct LineSplit {
    static constexpr int N1 = M == 128 ? 16 : 8;
    static constexpr int N2 = M / N1;
};

// Stage 1 of one line: thread n2 transforms places N2 n1 + n2 (read through
// `at`, a pointer to place p) and returns result k1, twiddled, in
// a[dft_at<N1>(k1)].
template <int M, bool INV, typename At>
__device__ __forceinline__ void line_stage1(double2 (&a)[LineSplit<M>::N1], int n2, At at,
                                            const double2* tw)
{
    constexpr int N1 = LineSplit<M>::N1, N2 = LineSplit<M>::N2, TS = 128 / M;
#pragma unroll
    for (int n1 = 0; n1 < N1; n1++) a[n1] = *at(N2 * n1 + n2);
    dft_small<N1, INV>(a);
#pragma unroll
    for (int k1 = 1; k1 < N1; k1++) {
        const double2 w = tw[(n2 * k1 * TS) & 127];
        a[dft_at<N1>(k1)] = c_mul(a[dft_at<N1>(k1)], INV ? c_conj(w) : w);
    }
}

// Copy of `total` elements by `nt` threads, B per thread in flight: all
// loads of a batch are issued before its stores.
template <int B, typename Load, typename Store>
__device__ __forceinline__ void batched_copy(int total, int t, int nt, Load ld, Store st)
{
    for (int base = 0; base < total; base += B * nt) {
        double2 v[B];
#pragma unroll
        for (int r = 0; r < B; r++) {
            const int i = base + r * nt + t;
            if (i < total) v[r] = ld(i);
        }
#pragma unroll
        for (int r = 0; r < B; r++) {
            const int i = base + r * nt + t;
            if (i < total) st(i, v[r]);
        }
    }
}

// Shared-memory place of plane row r, column c ([M][M/2+1]), with a spare
// entry after every 8 rows so that rows 8 apart fall in different banks.
__device__ __forceinline__ int pl_at(int r, int c, int MH) { return r * MH + (r >> 3) + c; }

template <int M>
constexpr size_t fft_plane_smem()
{
    return sizeof(double2) * ((size_t)M * (M / 2 + 1) + M / 8);
}

// Place k of z-line pair y (the complex line r_y + i r_(y + M/2)) in the
// plane: k <= M/2 in row y, the others in row y + M/2 at M - k, so that the
// unpacking reads C[k] and C[M - k] from the two places it writes.
__device__ __forceinline__ int zl_at(int y, int k, int M, int MH)
{
    return k <= M / 2 ? pl_at(y, k, MH) : pl_at(y + M / 2, M - k, MH);
}

// The columns kz of the plane along y, in place (rows = places).
template <int M, bool INV>
__device__ __forceinline__ void plane_columns(double2* plane, const double2* tw, int t)
{
    constexpr int MH = M / 2 + 1, N1 = LineSplit<M>::N1, N2 = LineSplit<M>::N2;
    constexpr int T1 = MH * N2, T2 = MH * N1;
    for (int base = 0; base < T1; base += FFT_THREADS) {
        const int task = base + t;
        if (task < T1) {
            const int kz = task / N2, n2 = task - kz * N2;
            double2 a[N1];
            auto at = [&](int p) { return plane + pl_at(p, kz, MH); };
            line_stage1<M, INV>(a, n2, at, tw);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++) *at(N2 * k1 + n2) = a[dft_at<N1>(k1)];
        }
    }
    __syncthreads();
    for (int base = 0; base < T2; base += FFT_THREADS) {
        const int task = base + t;
        double2 c[N2];
        int kz = 0, k1 = 0;
        if (task < T2) {
            kz = task / N1;
            k1 = task - kz * N1;
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) c[n2] = plane[pl_at(N2 * k1 + n2, kz, MH)];
            dft_small<N2, INV>(c);
        }
        __syncthreads();
        if (task < T2) {
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) plane[pl_at(k1 + N1 * k2, kz, MH)] = c[k2];
        }
        __syncthreads();
    }
}

template <int M>
__global__ void __launch_bounds__(FFT_THREADS) k_fft_zy(const SysDev* __restrict__ sys,
                                                        const int* __restrict__ order, int first,
                                                        const double* __restrict__ grid,
                                                        double2* __restrict__ spec,
                                                        const double2* __restrict__ twg)
{
    constexpr int MH = M / 2 + 1, N1 = LineSplit<M>::N1, N2 = LineSplit<M>::N2;
    constexpr int T1 = (M / 2) * N2, T2 = (M / 2) * N1;
    extern __shared__ double2 plane[];   // [M][MH], pl_at
    __shared__ double2 tw[128];
    const int t = threadIdx.x;
    const SysDev& S = sys[order[first + blockIdx.x / M]];
    const int x = blockIdx.x % M;
    const double* gp = grid + S.grid_off + (long long)x * M * M;
    for (int i = t; i < 128; i += FFT_THREADS) tw[i] = twg[i];
    __syncthreads();

    // z lines in pairs (y, y + M/2), c = r_y + i r_y': stage 1 from the grid
    for (int base = 0; base < T1; base += FFT_THREADS) {
        const int task = base + t;
        if (task < T1) {
            const int y = task / N2, n2 = task - y * N2;
            double2 a[N1];
            const double* r0 = gp + (long long)y * M;
            const double* r1 = r0 + (long long)(M / 2) * M;
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++)
                a[n1] = make_double2(r0[N2 * n1 + n2], r1[N2 * n1 + n2]);
            dft_small<N1, false>(a);
#pragma unroll
            for (int k1 = 1; k1 < N1; k1++)
                a[dft_at<N1>(k1)] = c_mul(a[dft_at<N1>(k1)], tw[(n2 * k1 * (128 / M)) & 127]);
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++)
                plane[zl_at(y, N2 * k1 + n2, M, MH)] = a[dft_at<N1>(k1)];
        }
    }
    __syncthreads();
    for (int base = 0; base < T2; base += FFT_THREADS) {
        const int task = base + t;
        double2 c[N2];
        int y = 0, k1 = 0;
        if (task < T2) {
            y = task / N1;
            k1 = task - y * N1;
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) c[n2] = plane[zl_at(y, N2 * k1 + n2, M, MH)];
            dft_small<N2, false>(c);
        }
        __syncthreads();
        if (task < T2) {
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) plane[zl_at(y, k1 + N1 * k2, M, MH)] = c[k2];
        }
        __syncthreads();
    }
    // unpack: R_y[k] = (C[k] + conj C[M-k]) / 2, R_y'[k] = (C[k] - conj C[M-k]) / 2i
    for (int i = t; i < (M / 2) * MH; i += FFT_THREADS) {
        const int y = i / MH, k = i - y * MH;
        const double2 a = plane[zl_at(y, k, M, MH)];
        const double2 b = c_conj(plane[zl_at(y, (M - k) & (M - 1), M, MH)]);
        plane[pl_at(y, k, MH)] = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y + b.y));
        plane[pl_at(y + M / 2, k, MH)] = make_double2(0.5 * (a.y - b.y), -0.5 * (a.x - b.x));
    }
    __syncthreads();
    plane_columns<M, false>(plane, tw, t);
    double2* sp = spec + S.spec_off + (long long)x * M * MH;
    for (int i = t; i < M * MH; i += FFT_THREADS) {
        const int r = i / MH;
        sp[i] = plane[pl_at(r, i - r * MH, MH)];
    }
}

// kz columns per CTA of the x pass: the M/2+1 columns of a ky in
// fft_x_blocks equal runs
template <int M>
constexpr int fft_x_blocks() { return (M / 2 + 1 + 15) / 16; }
template <int M>
constexpr int fft_x_cols() { return (M / 2 + 1 + fft_x_blocks<M>() - 1) / fft_x_blocks<M>(); }
constexpr int FFT_X_THREADS = 256;

template <int M>
__global__ void __launch_bounds__(FFT_X_THREADS, 2) k_fft_x_scale(const SysDev* __restrict__ sys,
                                                               const int* __restrict__ order,
                                                               int first,
                                                               double2* __restrict__ spec,
                                                               const double2* __restrict__ twg)
{
    constexpr int MH = M / 2 + 1, NB = fft_x_blocks<M>(), KB = fft_x_cols<M>();
    constexpr int N1 = LineSplit<M>::N1, N2 = LineSplit<M>::N2;
    constexpr int T1 = KB * N2, T2 = KB * N1;
    static_assert(T1 <= FFT_X_THREADS && T2 <= FFT_X_THREADS, "one task per thread");
    __shared__ double2 tw[128];
    __shared__ double2 lines[M * KB];   // place p of line c at p * KB + c
    __shared__ double ez[M];            // exp(scalar k^2) of each wave number index
    const int t = threadIdx.x;
    const int per_sys = M * NB;
    const SysDev& S = sys[order[first + blockIdx.x / per_sys]];
    const int rem = blockIdx.x % per_sys, ky = rem / NB, kz0 = (rem % NB) * KB;
    const int nkz = min(KB, MH - kz0);
    double2* sp = spec + S.spec_off;
    for (int i = t; i < 128; i += FFT_X_THREADS) tw[i] = twg[i];
    for (int i = t; i < M; i += FFT_X_THREADS) {
        const double k = kwave(i, M, S.kfac);
        ez[i] = exp(S.scalar * (k * k));
    }
    batched_copy<8>(
        M * KB, t, FFT_X_THREADS,
        [&](int i) {
            const int xx = i / KB, c = i - xx * KB;
            return c < nkz ? sp[((long long)xx * M + ky) * MH + kz0 + c] : make_double2(0.0, 0.0);
        },
        [&](int i, double2 v) { lines[i] = v; });
    __syncthreads();
    const double kyv = kwave(ky, M, S.kfac);
#pragma unroll 1
    for (int pass = 0; pass < 2; pass++) {   // forward (times Z), then inverse
        const bool inv = pass == 1;
        if (t < T1) {
            const int c = t / N2, n2 = t - c * N2;
            if (c < nkz) {
                double2 a[N1];
                auto at = [&](int p) { return lines + p * KB + c; };
                if (inv) line_stage1<M, true>(a, n2, at, tw);
                else line_stage1<M, false>(a, n2, at, tw);
#pragma unroll
                for (int k1 = 0; k1 < N1; k1++) *at(N2 * k1 + n2) = a[dft_at<N1>(k1)];
            }
        }
        __syncthreads();
        double2 cc[N2];
        const int c = t / N1, k1 = t - (t / N1) * N1;
        const bool act = t < T2 && c < nkz;
        if (act) {
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) cc[n2] = lines[(N2 * k1 + n2) * KB + c];
            if (inv) {
                dft_small<N2, true>(cc);
            } else {
                dft_small<N2, false>(cc);
                // Z as the scaling pass applies it: exp(scalar K^2) / K^2 * 4 pi / M^3,
                // the exponential as the product of the three axes' factors
                const int kz = kz0 + c;
                const double kzv = kwave(kz, M, S.kfac);
#pragma unroll
                for (int k2 = 0; k2 < N2; k2++) {
                    const int kx = k1 + N1 * k2;
                    const double kxv = kwave(kx, M, S.kfac);
                    const double K2 = (kzv * kzv + kyv * kyv) + kxv * kxv;
                    const double Z = (kx == 0 && ky == 0 && kz == 0)
                                         ? 0.0
                                         : ez[kx] * ez[ky] * ez[kz] / K2 * S.dnorm;
                    cc[k2].x *= Z;
                    cc[k2].y *= Z;
                }
            }
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) lines[(k1 + N1 * k2) * KB + c] = cc[k2];
        }
        __syncthreads();
    }
    for (int i = t; i < M * KB; i += FFT_X_THREADS) {
        const int xx = i / KB, c = i - xx * KB;
        if (c < nkz) sp[((long long)xx * M + ky) * MH + kz0 + c] = lines[i];
    }
}

// grid32: the FP32 copy of the grids, written beside the FP64 grid when set.
template <int M>
__global__ void __launch_bounds__(FFT_THREADS) k_ifft_yz(const SysDev* __restrict__ sys,
                                                         const int* __restrict__ order, int first,
                                                         const double2* __restrict__ spec,
                                                         double* __restrict__ grid,
                                                         float* __restrict__ grid32,
                                                         const double2* __restrict__ twg)
{
    constexpr int MH = M / 2 + 1, N1 = LineSplit<M>::N1, N2 = LineSplit<M>::N2;
    constexpr int T1 = (M / 2) * N2, T2 = (M / 2) * N1;
    static_assert(T1 <= FFT_THREADS, "the z-line stage 1 reads every pair in one round");
    extern __shared__ double2 plane[];   // [M][MH], pl_at
    __shared__ double2 tw[128];
    const int t = threadIdx.x;
    const SysDev& S = sys[order[first + blockIdx.x / M]];
    const int x = blockIdx.x % M;
    const double2* sp = spec + S.spec_off + (long long)x * M * MH;
    for (int i = t; i < 128; i += FFT_THREADS) tw[i] = twg[i];
    batched_copy<8>(
        M * MH, t, FFT_THREADS, [&](int i) { return sp[i]; },
        [&](int i, double2 v) {
            const int r = i / MH;
            plane[pl_at(r, i - r * MH, MH)] = v;
        });
    __syncthreads();
    plane_columns<M, true>(plane, tw, t);
    // z lines in pairs: C = R_y + i R_y' from the Hermitian half spectra;
    // stage 1 reads every pair before any place is overwritten
    for (int base = 0; base < T1; base += FFT_THREADS) {
        const int task = base + t;
        double2 a[N1];
        int y = 0, n2 = 0;
        if (task < T1) {
            y = task / N2;
            n2 = task - y * N2;
            auto at = [&](int k) {
                const bool low = k <= M / 2;
                const int kk = low ? k : M - k;
                double2 u = plane[pl_at(y, kk, MH)], v = plane[pl_at(y + M / 2, kk, MH)];
                if (!low) {
                    u = c_conj(u);
                    v = c_conj(v);
                }
                return make_double2(u.x - v.y, u.y + v.x);
            };
#pragma unroll
            for (int n1 = 0; n1 < N1; n1++) a[n1] = at(N2 * n1 + n2);
            dft_small<N1, true>(a);
#pragma unroll
            for (int k1 = 1; k1 < N1; k1++)
                a[dft_at<N1>(k1)] =
                    c_mul(a[dft_at<N1>(k1)], c_conj(tw[(n2 * k1 * (128 / M)) & 127]));
        }
        __syncthreads();
        if (task < T1) {
#pragma unroll
            for (int k1 = 0; k1 < N1; k1++)
                plane[zl_at(y, N2 * k1 + n2, M, MH)] = a[dft_at<N1>(k1)];
        }
    }
    __syncthreads();
    // stage 2: c[n] = r_y[n] + i r_y'[n] straight to the grid rows
    const long long goff = S.grid_off + (long long)x * M * M;
    for (int base = 0; base < T2; base += FFT_THREADS) {
        const int task = base + t;
        if (task < T2) {
            const int y = task / N1, k1 = task - y * N1;
            double2 c[N2];
#pragma unroll
            for (int n2 = 0; n2 < N2; n2++) c[n2] = plane[zl_at(y, N2 * k1 + n2, M, MH)];
            dft_small<N2, true>(c);
#pragma unroll
            for (int k2 = 0; k2 < N2; k2++) {
                const long long i0 = goff + (long long)y * M + k1 + N1 * k2;
                const long long i1 = i0 + (long long)(M / 2) * M;
                grid[i0] = c[k2].x;
                grid[i1] = c[k2].y;
                if (grid32) {
                    grid32[i0] = (float)c[k2].x;
                    grid32[i1] = (float)c[k2].y;
                }
            }
        }
    }
}
