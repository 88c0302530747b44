// Field solver: right-hand sides, then every DST-I / DCT-I / mixed transform
// pair of compute_fields (lcode/plasma3d/fields.py:176-322) as four waves of
// one batched dense matrix product each, then the finishing epilogues.
//
// Seven problems per call, in this order (n = N - 2):
//   0 Ey, 1 Bx : X = rhs[1:-1, :]   (n x N); out = S (M  o (S X C^T)) C^T
//   2 Ex, 3 By : X = rhs[:, 1:-1]   (N x n); out = C (M^T o (C X S)) S
//   4 Ez, 5 Phi: X = rhs[1:-1,1:-1] (n x n); out = S (D  o (S X S)) S
//   6 Bz       : X = rhs            (N x N); out = C (Nm o (C X C^T)) C^T
// with S the DST-I matrix, C the DCT-I matrix, M the mixed, D the Dirichlet
// and Nm the Neumann solver matrices (initialization.py:15-67).  The
// transposed fields Ex, By follow from mix2d(X^T)^T = C X S.
//
// Waves: (1) T = X R, (2) U = (L T) o Mat, (3) T = U R, (4) out = L T with the
// field epilogue (half/full combination, zero border), then Bz's mean removal.
#include "common.cuh"

namespace lcb {

constexpr int NPROB = 7;

template <typename T>
struct GemmDesc {
    const T *A; const T *B; T *C;
    const T *E;        // spectral matrix for EPI_SCALE
    int lda, ldb, ldc, lde;
    int M, N, K;
};

enum Epi { EPI_STORE = 0, EPI_SCALE = 1, EPI_FIELD = 2 };

// Field epilogue of wave 4 for one problem: destination offsets and kind.
struct FieldOut {
    double *half, *full;      // may be NULL
    const double *prev;       // fields_prev plane
    int row_off, col_off;     // position of the (M x N) block in the N x N plane
    int kind;                 // 0 transverse (half=v, full=2v-prev), 1 Ez, 2 Phi, 3 Bz raw
    double *bz_raw;           // kind 3: raw plane (N x N, compact)
    double *bz_sum;           // kind 3: accumulated sum
};

template <typename T>
struct GemmBatch {
    GemmDesc<T> d[NPROB];
    FieldOut out[NPROB];
    int grid_n;   // plane size N (for field epilogue)
};

// ---------------------------------------------------------------------------
// Batched NN GEMM, C = A (MxK) * B (KxN), row-major, one problem per
// blockIdx.z.  BM x BN tile per CTA, TM x TN outputs per thread, BK-deep
// k-slices staged in shared memory (A stored k-major for broadcast reads).
// ---------------------------------------------------------------------------
template <typename T, int BM, int BN, int BK, int TM, int TN, int EPI>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
k_gemm_batched(const __grid_constant__ GemmBatch<T> batch)
{
    constexpr int NT = (BM / TM) * (BN / TN);
    const GemmDesc<T> &g = batch.d[blockIdx.z];
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    if (m0 >= g.M || n0 >= g.N) return;

    __shared__ T As[2][BK][BM + 1];
    __shared__ T Bs[2][BK][BN];

    const int tid = threadIdx.x;
    const int tn = tid % (BN / TN), tm = tid / (BN / TN);
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] = T(0);

    constexpr int A_PER = (BM * BK + NT - 1) / NT;
    constexpr int B_PER = (BK * BN + NT - 1) / NT;
    T ra[A_PER], rb[B_PER];

    auto load_regs = [&](int k0) {
#pragma unroll
        for (int r = 0; r < A_PER; r++) {
            const int e = tid + r * NT;
            const int mm = e / BK, kk = e % BK;
            const int gm = m0 + mm, gk = k0 + kk;
            ra[r] = (e < BM * BK && gm < g.M && gk < g.K) ? g.A[(int64_t)gm * g.lda + gk] : T(0);
        }
#pragma unroll
        for (int r = 0; r < B_PER; r++) {
            const int e = tid + r * NT;
            const int kk = e / BN, nn = e % BN;
            const int gk = k0 + kk, gn = n0 + nn;
            rb[r] = (e < BK * BN && gk < g.K && gn < g.N) ? g.B[(int64_t)gk * g.ldb + gn] : T(0);
        }
    };
    auto store_smem = [&](int buf) {
#pragma unroll
        for (int r = 0; r < A_PER; r++) {
            const int e = tid + r * NT;
            if (e < BM * BK) As[buf][e % BK][e / BK] = ra[r];
        }
#pragma unroll
        for (int r = 0; r < B_PER; r++) {
            const int e = tid + r * NT;
            if (e < BK * BN) Bs[buf][e / BN][e % BN] = rb[r];
        }
    };

    const int nk = (g.K + BK - 1) / BK;
    load_regs(0);
    store_smem(0);
    __syncthreads();
    for (int kt = 0; kt < nk; kt++) {
        const int buf = kt & 1;
        if (kt + 1 < nk) load_regs((kt + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            T a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; i++) a[i] = As[buf][kk][tm * TM + i];
#pragma unroll
            for (int j = 0; j < TN; j++) b[j] = Bs[buf][kk][tn + j * (BN / TN)];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[i][j] += a[i] * b[j];
        }
        if (kt + 1 < nk) store_smem(buf ^ 1);
        __syncthreads();
    }

    // ---- epilogue ----
    double part_sum = 0;
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int gm = m0 + tm * TM + i;
        if (gm >= g.M) continue;
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const int gn = n0 + tn + j * (BN / TN);
            if (gn >= g.N) continue;
            const T v = acc[i][j];
            if (EPI == EPI_STORE) {
                g.C[(int64_t)gm * g.ldc + gn] = v;
            } else if (EPI == EPI_SCALE) {
                g.C[(int64_t)gm * g.ldc + gn] = v * g.E[(int64_t)gm * g.lde + gn];
            } else {
                const FieldOut &o = batch.out[blockIdx.z];
                const int64_t off = (int64_t)(gm + o.row_off) * batch.grid_n + gn + o.col_off;
                const double dv = (double)v;
                if (o.kind == 0) {
                    if (o.half) o.half[off] = dv;
                    if (o.full) o.full[off] = 2 * dv - o.prev[off];
                } else if (o.kind == 1) {
                    if (o.full) o.full[off] = dv;
                    if (o.half) o.half[off] = (dv + o.prev[off]) / 2;
                } else if (o.kind == 2) {
                    if (o.full) o.full[off] = dv;
                    if (o.half) o.half[off] = dv;
                } else {
                    o.bz_raw[off] = dv;
                    part_sum += dv;
                }
            }
        }
    }
    if (EPI == EPI_FIELD && batch.out[blockIdx.z].kind == 3) {
        // block reduction of the Bz partial sums, one atomic per CTA
        __shared__ double red[32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part_sum += __shfl_xor_sync(0xffffffffu, part_sum, o);
        if ((tid & 31) == 0) red[tid >> 5] = part_sum;
        __syncthreads();
        if (tid < 32) {
            double s = tid < NT / 32 ? red[tid] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (tid == 0) atomicAdd(batch.out[blockIdx.z].bz_sum, s);
        }
    }
}

// ---------------------------------------------------------------------------
// Right-hand sides (fields.py:112-230), one thread per grid node.
// ---------------------------------------------------------------------------
struct RhsArgs {
    int N;
    double h, dxi, c, rb_div;
    const double *ro_f, *jx_f, *jy_f, *jz_f;  // full currents, n_f planes
    const double *ro_p, *jx_p, *jy_p, *jz_p;  // prev currents, n_p planes
    int n_f, n_p;
    const double *rb_full, *rb_prev;
    const double *Ex, *Ey, *Bx, *By;          // fields (Helmholtz term)
    double *bz_sum;
};

__device__ __forceinline__ double sum_planes(const double *a, int np, int64_t plane, int64_t i)
{
    double s = a[i];
    for (int p = 1; p < np; p++) s += a[i + p * plane];
    return s;
}

template <typename T>
__global__ void __launch_bounds__(256)
k_fields_rhs(RhsArgs a, T *X0, T *X1, T *X2, T *X3, T *X4, T *X5, T *X6)
{
    const int N = a.N, n = N - 2;
    const int64_t plane = (int64_t)N * N;
    const int64_t total = plane;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        if (t == 0 && a.bz_sum) *a.bz_sum = 0.0;
        const int i = (int)(t / N), j = (int)(t % N);
        const bool inner = i >= 1 && i < N - 1 && j >= 1 && j < N - 1;
        // ro_half / jz_half = (full + rb_full + prev + rb_prev) / 2
        auto rho_half = [&](int64_t q) {
            const double rbf = a.rb_full[q] / a.rb_div, rbp = a.rb_prev[q] / a.rb_div;
            return (sum_planes(a.ro_f, a.n_f, plane, q) + rbf +
                    sum_planes(a.ro_p, a.n_p, plane, q) + rbp) / 2;
        };
        auto jz_half = [&](int64_t q) {
            const double rbf = a.rb_full[q] / a.rb_div, rbp = a.rb_prev[q] / a.rb_div;
            return (sum_planes(a.jz_f, a.n_f, plane, q) + rbf +
                    sum_planes(a.jz_p, a.n_p, plane, q) + rbp) / 2;
        };
        double dro_dx = 0, dro_dy = 0, djz_dx = 0, djz_dy = 0;
        if (inner) {
            dro_dx = (rho_half(t + N) - rho_half(t - N)) / (a.h * 2);
            dro_dy = (rho_half(t + 1) - rho_half(t - 1)) / (a.h * 2);
            djz_dx = (jz_half(t + N) - jz_half(t - N)) / (a.h * 2);
            djz_dy = (jz_half(t + 1) - jz_half(t - 1)) / (a.h * 2);
        }
        const double jx_full = sum_planes(a.jx_f, a.n_f, plane, t);
        const double jy_full = sum_planes(a.jy_f, a.n_f, plane, t);
        const double djx_dxi = (sum_planes(a.jx_p, a.n_p, plane, t) - jx_full) / a.dxi;
        const double djy_dxi = (sum_planes(a.jy_p, a.n_p, plane, t) - jy_full) / a.dxi;
        const double Ex_rhs = -(dro_dx - djx_dxi - a.c * a.Ex[t]);
        const double Ey_rhs = -(dro_dy - djy_dxi - a.c * a.Ey[t]);
        const double Bx_rhs = +(djz_dy - djy_dxi + a.c * a.Bx[t]);
        const double By_rhs = -(djz_dx - djx_dxi - a.c * a.By[t]);
        // Ey, Bx: rows 1..N-2, all columns -> (n x N)
        if (i >= 1 && i < N - 1) {
            const int64_t o = (int64_t)(i - 1) * N + j;
            X0[o] = (T)Ey_rhs;
            X1[o] = (T)Bx_rhs;
        }
        // Ex, By: all rows, columns 1..N-2 -> (N x n)
        if (j >= 1 && j < N - 1) {
            const int64_t o = (int64_t)i * n + (j - 1);
            X2[o] = (T)Ex_rhs;
            X3[o] = (T)By_rhs;
        }
        // Bz rhs over the whole plane, differences zero on the perimeter
        double djx_dy = 0, djy_dx = 0;
        if (inner) {
            djx_dy = sum_planes(a.jx_f, a.n_f, plane, t + 1) - sum_planes(a.jx_f, a.n_f, plane, t - 1);
            djy_dx = sum_planes(a.jy_f, a.n_f, plane, t + N) - sum_planes(a.jy_f, a.n_f, plane, t - N);
        }
        X6[t] = (T)(-(djx_dy - djy_dx) / (a.h * 2));
        if (inner) {
            const int64_t o = (int64_t)(i - 1) * n + (j - 1);
            const double djx_dx = sum_planes(a.jx_f, a.n_f, plane, t + N) - sum_planes(a.jx_f, a.n_f, plane, t - N);
            const double djy_dy = sum_planes(a.jy_f, a.n_f, plane, t + 1) - sum_planes(a.jy_f, a.n_f, plane, t - 1);
            X4[o] = (T)(-(djx_dx + djy_dy) / (a.h * 2));
            X5[o] = (T)(sum_planes(a.ro_f, a.n_f, plane, t) - sum_planes(a.jz_f, a.n_f, plane, t));
        }
    }
}

// Bz mean removal and half average, plus the zero borders of every output
// plane (the reference pads its inner solutions with zeros).
struct FinishArgs {
    int N;
    const double *bz_raw, *bz_sum, *bz_prev;
    double *bz_full, *bz_half;
    double *half[7], *full[7];
    const double *prev[7];
};

__global__ void __launch_bounds__(256) k_fields_finish(FinishArgs a)
{
    const int N = a.N;
    const int64_t plane = (int64_t)N * N;
    const double mean = *a.bz_sum / (double)plane;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < plane;
         t += (int64_t)gridDim.x * blockDim.x) {
        const double v = a.bz_raw[t] - mean;
        if (a.bz_full) a.bz_full[t] = v;
        if (a.bz_half) a.bz_half[t] = (v + a.bz_prev[t]) / 2;
        const int i = (int)(t / N), j = (int)(t % N);
        const bool row_edge = (i == 0 || i == N - 1), col_edge = (j == 0 || j == N - 1);
        // The solutions are zero on their Dirichlet edges: Ex(0), By(4) on the
        // first/last column, Ey(1), Bx(3) on the first/last row, Ez(2), Phi(6)
        // on all four.  There the reference's combinations reduce to
        // full = 2*0 - prev (transverse), Ez half = (0 + prev)/2, Phi = 0.
        const bool edge[7] = {col_edge, row_edge, row_edge || col_edge, row_edge,
                              col_edge, false, row_edge || col_edge};
#pragma unroll
        for (int f = 0; f < 7; f++) {
            if (!edge[f] || f == 5) continue;
            const bool transverse = (f == 0 || f == 1 || f == 3 || f == 4);
            if (a.half[f]) a.half[f][t] = (f == 2) ? (0.0 + a.prev[f][t]) / 2 : 0.0;
            if (a.full[f]) a.full[f][t] = transverse ? 2 * 0.0 - a.prev[f][t] : 0.0;
        }
    }
}

template <typename T>
struct Work {
    T *X[NPROB], *Tm[NPROB];
    double *bz_raw, *bz_sum;
};

static size_t plane_elems(int N) { return (size_t)N * N; }

template <typename T>
static size_t work_bytes(int N)
{
    size_t b = 2 * NPROB * plane_elems(N) * sizeof(T);
    b = (b + 255) / 256 * 256;
    b += plane_elems(N) * sizeof(double);
    b = (b + 255) / 256 * 256;
    b += 256;
    return b;
}

template <typename T>
static Work<T> carve(void *ws, int N)
{
    Work<T> w;
    T *p = static_cast<T *>(ws);
    for (int i = 0; i < NPROB; i++) { w.X[i] = p; p += plane_elems(N); }
    for (int i = 0; i < NPROB; i++) { w.Tm[i] = p; p += plane_elems(N); }
    size_t off = 2 * NPROB * plane_elems(N) * sizeof(T);
    off = (off + 255) / 256 * 256;
    char *base = static_cast<char *>(ws);
    w.bz_raw = reinterpret_cast<double *>(base + off);
    off += plane_elems(N) * sizeof(double);
    off = (off + 255) / 256 * 256;
    w.bz_sum = reinterpret_cast<double *>(base + off);
    return w;
}

template <typename T, int BM, int BN, int BK, int TM, int TN>
static int launch_wave(const GemmBatch<T> &b, int epi, cudaStream_t st, const char *what)
{
    int maxM = 0, maxN = 0;
    for (int p = 0; p < NPROB; p++) {
        maxM = b.d[p].M > maxM ? b.d[p].M : maxM;
        maxN = b.d[p].N > maxN ? b.d[p].N : maxN;
    }
    dim3 grid((maxN + BN - 1) / BN, (maxM + BM - 1) / BM, NPROB);
    constexpr int NT = (BM / TM) * (BN / TN);
    if (epi == EPI_STORE)
        k_gemm_batched<T, BM, BN, BK, TM, TN, EPI_STORE><<<grid, NT, 0, st>>>(b);
    else if (epi == EPI_SCALE)
        k_gemm_batched<T, BM, BN, BK, TM, TN, EPI_SCALE><<<grid, NT, 0, st>>>(b);
    else
        k_gemm_batched<T, BM, BN, BK, TM, TN, EPI_FIELD><<<grid, NT, 0, st>>>(b);
    LCB_LAUNCH_CHECK(what);
    return LCB_OK;
}

template <typename T>
static int run_wave(const GemmBatch<T> &b, int epi, int N, cudaStream_t st, const char *what)
{
    if (N > 160) return launch_wave<T, 64, 64, 16, 4, 4>(b, epi, st, what);
    return launch_wave<T, 32, 32, 16, 2, 2>(b, epi, st, what);
}

template <typename T>
struct Ops {
    const T *S, *C, *CT, *D, *Mx, *MxT, *Nm;
};

template <typename T>
static int solve(const lcb_compute_fields_args *a, const Ops<T> &op, cudaStream_t st)
{
    const int N = a->grid_steps, n = N - 2;
    Work<T> w = carve<T>(a->workspace, N);

    RhsArgs r;
    r.N = N; r.h = a->h; r.dxi = a->xi_step; r.c = a->subtraction_coeff;
    r.rb_div = a->rho_beam_divisor;
    r.ro_f = a->currents_full.ro; r.jx_f = a->currents_full.jx;
    r.jy_f = a->currents_full.jy; r.jz_f = a->currents_full.jz;
    r.n_f = a->currents_full.n_planes;
    r.ro_p = a->currents_prev.ro; r.jx_p = a->currents_prev.jx;
    r.jy_p = a->currents_prev.jy; r.jz_p = a->currents_prev.jz;
    r.n_p = a->currents_prev.n_planes;
    r.rb_full = a->rho_beam_full; r.rb_prev = a->rho_beam_prev;
    r.Ex = a->fields.f[0]; r.Ey = a->fields.f[1];
    r.Bx = a->fields.f[3]; r.By = a->fields.f[4];
    r.bz_sum = w.bz_sum;
    {
        const int64_t tot = (int64_t)N * N;
        int blocks = (int)((tot + 255) / 256);
        k_fields_rhs<T><<<blocks, 256, 0, st>>>(r, w.X[0], w.X[1], w.X[2], w.X[3],
                                               w.X[4], w.X[5], w.X[6]);
        LCB_LAUNCH_CHECK("k_fields_rhs");
    }

    // Per-problem shapes: rows x cols of X, and the left / right operators.
    const int rows[NPROB] = {n, n, N, N, n, n, N};
    const int cols[NPROB] = {N, N, n, n, n, n, N};
    const T *Lop[NPROB] = {op.S, op.S, op.C, op.C, op.S, op.S, op.C};
    const T *Rop[NPROB] = {op.CT, op.CT, op.S, op.S, op.S, op.S, op.CT};
    const T *Mat[NPROB] = {op.Mx, op.Mx, op.MxT, op.MxT, op.D, op.D, op.Nm};

    GemmBatch<T> b;
    memset(&b, 0, sizeof(b));
    b.grid_n = N;
    // wave 1: Tm = X * R
    for (int p = 0; p < NPROB; p++) {
        GemmDesc<T> &d = b.d[p];
        d.A = w.X[p]; d.lda = cols[p];
        d.B = Rop[p]; d.ldb = cols[p];
        d.C = w.Tm[p]; d.ldc = cols[p];
        d.M = rows[p]; d.N = cols[p]; d.K = cols[p];
    }
    int rc = run_wave<T>(b, EPI_STORE, N, st, "wave1");
    if (rc) return rc;
    // wave 2: X = (L * Tm) o Mat
    for (int p = 0; p < NPROB; p++) {
        GemmDesc<T> &d = b.d[p];
        d.A = Lop[p]; d.lda = rows[p];
        d.B = w.Tm[p]; d.ldb = cols[p];
        d.C = w.X[p]; d.ldc = cols[p];
        d.E = Mat[p]; d.lde = cols[p];
        d.M = rows[p]; d.N = cols[p]; d.K = rows[p];
    }
    rc = run_wave<T>(b, EPI_SCALE, N, st, "wave2");
    if (rc) return rc;
    // wave 3: Tm = X * R
    for (int p = 0; p < NPROB; p++) {
        GemmDesc<T> &d = b.d[p];
        d.A = w.X[p]; d.lda = cols[p];
        d.B = Rop[p]; d.ldb = cols[p];
        d.C = w.Tm[p]; d.ldc = cols[p];
        d.E = nullptr;
        d.M = rows[p]; d.N = cols[p]; d.K = cols[p];
    }
    rc = run_wave<T>(b, EPI_STORE, N, st, "wave3");
    if (rc) return rc;
    // wave 4: out = L * Tm, field epilogues
    // field index in lcb_fields: Ex 0, Ey 1, Ez 2, Bx 3, By 4, Bz 5, Phi 6
    const int fidx[NPROB] = {1, 3, 0, 4, 2, 6, 5};
    const int roff[NPROB] = {1, 1, 0, 0, 1, 1, 0};
    const int coff[NPROB] = {0, 0, 1, 1, 1, 1, 0};
    const int kind[NPROB] = {0, 0, 0, 0, 1, 2, 3};
    for (int p = 0; p < NPROB; p++) {
        GemmDesc<T> &d = b.d[p];
        d.A = Lop[p]; d.lda = rows[p];
        d.B = w.Tm[p]; d.ldb = cols[p];
        d.C = nullptr; d.ldc = 0;
        d.M = rows[p]; d.N = cols[p]; d.K = rows[p];
        FieldOut &o = b.out[p];
        const int f = fidx[p];
        o.half = a->out_half.f[f]; o.full = a->out_full.f[f];
        o.prev = a->fields_prev.f[f];
        o.row_off = roff[p]; o.col_off = coff[p]; o.kind = kind[p];
        o.bz_raw = w.bz_raw; o.bz_sum = w.bz_sum;
    }
    rc = run_wave<T>(b, EPI_FIELD, N, st, "wave4");
    if (rc) return rc;

    FinishArgs fa;
    fa.N = N; fa.bz_raw = w.bz_raw; fa.bz_sum = w.bz_sum;
    fa.bz_prev = a->fields_prev.f[5];
    fa.bz_full = a->out_full.f[5]; fa.bz_half = a->out_half.f[5];
    for (int f = 0; f < 7; f++) {
        fa.half[f] = a->out_half.f[f];
        fa.full[f] = a->out_full.f[f];
        fa.prev[f] = a->fields_prev.f[f];
    }
    {
        const int64_t tot = (int64_t)N * N;
        int blocks = (int)((tot + 255) / 256);
        k_fields_finish<<<blocks, 256, 0, st>>>(fa);
        LCB_LAUNCH_CHECK("k_fields_finish");
    }
    return LCB_OK;
}

}  // namespace lcb

using namespace lcb;

extern "C" size_t lcb_compute_fields_workspace_bytes(int grid_steps, int precision)
{
    if (grid_steps < 5) return 0;
    return precision == LCB_PREC_MIXED ? work_bytes<float>(grid_steps)
                                       : work_bytes<double>(grid_steps);
}

extern "C" int lcb_compute_fields(const lcb_compute_fields_args *a, void *stream)
{
    LCB_REQUIRE(a, "args is NULL");
    const int N = a->grid_steps;
    LCB_REQUIRE(N >= 5 && (N % 2) == 1, "grid_steps must be odd and >= 5 (got %d)", N);
    LCB_REQUIRE(a->workspace && a->workspace_bytes >= lcb_compute_fields_workspace_bytes(N, a->precision),
                "compute_fields workspace too small (%zu < %zu)", a->workspace_bytes,
                lcb_compute_fields_workspace_bytes(N, a->precision));
    LCB_REQUIRE(((uintptr_t)a->workspace & 255) == 0, "workspace must be 256-byte aligned");
    LCB_REQUIRE(a->currents_full.n_planes >= 1 && a->currents_full.n_planes <= 2 &&
                a->currents_prev.n_planes >= 1 && a->currents_prev.n_planes <= 2,
                "currents must have 1 or 2 planes");
    LCB_REQUIRE(a->rho_beam_divisor != 0.0, "rho_beam_divisor is 0");
    for (int f : {0, 1, 3, 4}) LCB_REQUIRE(a->fields.f[f], "fields plane %d is NULL", f);
    for (int f = 0; f < 6; f++) LCB_REQUIRE(a->fields_prev.f[f], "fields_prev plane %d is NULL", f);
    cudaStream_t st = as_stream(stream);
    if (a->precision == LCB_PREC_MIXED) {
        const lcb_field_consts &c = a->consts;
        LCB_REQUIRE(c.dst_f && c.dct_f && c.dctT_f && c.dirichlet_f && c.mixed_f &&
                    c.mixedT_f && c.neumann_f, "FP32 operators missing");
        Ops<float> op{c.dst_f, c.dct_f, c.dctT_f, c.dirichlet_f, c.mixed_f, c.mixedT_f, c.neumann_f};
        return solve<float>(a, op, st);
    }
    LCB_REQUIRE(a->precision == LCB_PREC_FP64, "bad precision %d", a->precision);
    const lcb_field_consts &c = a->consts;
    LCB_REQUIRE(c.dst && c.dct && c.dctT && c.dirichlet && c.mixed && c.mixedT && c.neumann,
                "FP64 operators missing");
    Ops<double> op{c.dst, c.dct, c.dctT, c.dirichlet, c.mixed, c.mixedT, c.neumann};
    return solve<double>(a, op, st);
}

// ---------------------------------------------------------------------------
// Allocation-free variant: the scratch is a file-scope device array instead
// of a caller-provided workspace (see lcb_compute_fields_noalloc in lcb.h).
// ---------------------------------------------------------------------------
#include <mutex>

namespace lcb {

static __device__ __align__(256) unsigned char g_fields_scratch[LCB_NOALLOC_FIELDS_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
static void *g_scratch_addr[kMaxDevices] = {};
static std::mutex g_scratch_mu;

// Device address of g_fields_scratch on the current device, looked up once
// per device.  The host-side symbol is only a stand-in and must never be
// handed to a kernel.
static int scratch_address(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_check(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device ordinal %d out of range for the allocation-free path", dev);
        return LCB_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_fields_scratch);
        if (e != cudaSuccess) return cuda_check(e, "cudaGetSymbolAddress(g_fields_scratch)");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return LCB_OK;
}

}  // namespace lcb

extern "C" int lcb_compute_fields_noalloc(const lcb_compute_fields_args *a, void *stream)
{
    LCB_REQUIRE(a, "args is NULL");
    const size_t need = lcb_compute_fields_workspace_bytes(a->grid_steps, a->precision);
    LCB_REQUIRE(need > 0, "grid_steps must be odd and >= 5 (got %d)", a->grid_steps);
    LCB_REQUIRE(need <= LCB_NOALLOC_FIELDS_SCRATCH_BYTES,
                "grid_steps %d in precision %d needs %zu bytes of scratch; the "
                "allocation-free entry point has %zu (largest grid: 263 in FP64, "
                "361 in mixed precision) -- use lcb_compute_fields with a workspace",
                a->grid_steps, a->precision, need, (size_t)LCB_NOALLOC_FIELDS_SCRATCH_BYTES);
    void *scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    lcb_compute_fields_args b = *a;
    b.workspace = scratch;
    b.workspace_bytes = LCB_NOALLOC_FIELDS_SCRATCH_BYTES;
    return lcb_compute_fields(&b, stream);
}
