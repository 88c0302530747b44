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
// field epilogue (half/full combination), then Bz's mean removal and edges.
//
// One butterfly level halves every product.  Both operators of odd length L
// obey T[k][L-1-j] = (-1)^k T[k][j] and vanish at the middle column for odd
// k, so an even output row k needs only the folded sum x_j + x_{L-1-j}
// (j < mid, plus x_mid) and an odd row only the folded difference (j < mid):
//   y_{2r}   = sum_{j<=mid} T[2r][j]   (x_j + x_{L-1-j})   (x_mid alone)
//   y_{2r+1} = sum_{j< mid} T[2r+1][j] (x_j - x_{L-1-j})
// Each product therefore splits into an even and an odd half-size product.
// A light pass folds the data operand before each wave (sum block U, then
// difference block V); the products write their even/odd outputs back
// interleaved, so every result is in natural order again.
//
// FP64 products run on the FP64 tensor cores (mma.sync m8n8k4 .f64); FP32
// products (mixed precision) on the FP32 cores.
#include <cstring>

#include "common.cuh"

namespace lcb {

constexpr int NPROB = 7;
enum { P_EY = 0, P_BX, P_EX, P_BY, P_EZ, P_PHI, P_BZ };

// ---------------------------------------------------------------------------
// Operators: folded transform blocks and solver matrices, built on the device.
// For a transform T of odd length L (S with L = n, C with L = N), He = (L+1)/2,
// Ho = (L-1)/2:  Te[r][j] = T[2r][j] (He x He), To[r][j] = T[2r+1][j] (Ho x Ho),
// TeT, ToT their transposes.
// ---------------------------------------------------------------------------
enum { OP_SE, OP_SO, OP_SET, OP_SOT, OP_CE, OP_CO, OP_CET, OP_COT,
       OP_D, OP_MX, OP_MXT, OP_NM, OP_COUNT };

// Leading dimensions of the dense operands are padded to an even number of
// elements so that every row starts on a 16-byte boundary (cp.async chunks).
__host__ __device__ constexpr int ld2(int c) { return (c + 1) & ~1; }

struct OpLayout {
    int64_t off[OP_COUNT + 1];  // element offsets, 32-element aligned
    int64_t rows[OP_COUNT], cols[OP_COUNT], ld[OP_COUNT];
};

static OpLayout op_layout(int N)
{
    const int n = N - 2;
    const int se = (n + 1) / 2, so = (n - 1) / 2, ce = (N + 1) / 2, co = (N - 1) / 2;
    const int64_t r[OP_COUNT] = {se, so, se, so, ce, co, ce, co, n, n, N, N};
    const int64_t c[OP_COUNT] = {se, so, se, so, ce, co, ce, co, n, N, n, N};
    OpLayout L;
    int64_t o = 0;
    for (int i = 0; i < OP_COUNT; i++) {
        L.off[i] = o;
        L.rows[i] = r[i];
        L.cols[i] = c[i];
        // transform blocks feed cp.async; solver matrices are read elementwise
        L.ld[i] = i < OP_D ? ld2((int)c[i]) : c[i];
        o += (r[i] * L.ld[i] + 31) / 32 * 32;
    }
    L.off[OP_COUNT] = o;
    return L;
}

// 2 sin(pi (j+1)(k+1)/(n+1)) with the argument reduced exactly in integers.
__device__ double dst1(int k, int j, int n)
{
    const int64_t p = 2 * (int64_t)(n + 1);
    const int64_t t = ((int64_t)(j + 1) * (k + 1)) % p;
    return 2.0 * sinpi((double)t / (double)(n + 1));
}

// c_j cos(pi j k/(N-1)), c_0 = c_{N-1} = 1, else 2.
__device__ double dct1(int k, int j, int N)
{
    const int64_t p = 2 * (int64_t)(N - 1);
    const int64_t t = ((int64_t)j * k) % p;
    const double c = (j == 0 || j == N - 1) ? 1.0 : 2.0;
    return c * cospi((double)t / (double)(N - 1));
}

// lam_k = 4/h^2 sin^2(k pi / (2 (N-1)))   (initialization.py:22-24)
__device__ double lam(int k, int N, double h)
{
    const double s = sinpi((double)k / (2.0 * (N - 1)));
    return 4 / (h * h) * (s * s);
}

template <typename T>
__global__ void k_build_ops(int N, double h, double c, OpLayout L, T *buf)
{
    const int n = N - 2;
    const double norm = (2.0 * (N - 1)) * (2.0 * (N - 1));
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < L.off[OP_COUNT];
         e += (int64_t)gridDim.x * blockDim.x) {
        int b = 0;
        while (b < OP_COUNT - 1 && e >= L.off[b + 1]) b++;
        const int64_t loc = e - L.off[b];
        const int r = (int)(loc / L.ld[b]), q = (int)(loc % L.ld[b]);
        if (r >= L.rows[b] || q >= L.cols[b]) { buf[e] = T(0); continue; }
        double v = 0;
        switch (b) {
        case OP_SE: v = dst1(2 * r, q, n); break;
        case OP_SO: v = dst1(2 * r + 1, q, n); break;
        case OP_SET: v = dst1(2 * q, r, n); break;
        case OP_SOT: v = dst1(2 * q + 1, r, n); break;
        case OP_CE: v = dct1(2 * r, q, N); break;
        case OP_CO: v = dct1(2 * r + 1, q, N); break;
        case OP_CET: v = dct1(2 * q, r, N); break;
        case OP_COT: v = dct1(2 * q + 1, r, N); break;
        case OP_D: v = 1 / (lam(r + 1, N, h) + lam(q + 1, N, h)) / norm; break;
        case OP_MX: v = 1 / (lam(r + 1, N, h) + lam(q, N, h) + c) / norm; break;
        case OP_MXT: v = 1 / (lam(q + 1, N, h) + lam(r, N, h) + c) / norm; break;
        case OP_NM: v = (r == 0 && q == 0) ? 0.0 : 1 / (lam(r, N, h) + lam(q, N, h)) / norm; break;
        }
        buf[e] = (T)v;
    }
}

// ---------------------------------------------------------------------------
// Batched GEMM descriptors.  Every product is a plain row-major
// C (M x N) = A (M x K) * B (K x N); the even/odd folds are done by the
// fold passes below, so operands arrive ready to stream.
// ---------------------------------------------------------------------------
template <typename T>
struct GemmDesc {
    const T *A; const T *B;
    T *C; const T *E;     // STORE / SCALE output (natural layout) and scale matrix
    int lda, ldb, ldc, lde;
    int M, N, K;
    int rmul, radd, cmul, cadd;  // output element (m, n) -> (rmul m + radd, cmul n + cadd)
    int prob;             // problem id, for the field epilogue
};

enum Epi { EPI_STORE = 0, EPI_SCALE = 1, EPI_FIELD = 2 };

struct FieldOut {
    double *half, *full;      // may be NULL
    const double *prev;       // fields_prev plane
    int row_off, col_off;     // position of the block in the N x N plane
    int kind;                 // 0 transverse (half=v, full=2v-prev), 1 Ez, 2 Phi, 3 Bz raw
    double *bz_raw, *bz_sum;
};

constexpr int MAXSUB = 2 * NPROB;

template <typename T>
struct GemmBatch {
    GemmDesc<T> d[MAXSUB];
    FieldOut out[NPROB];
    int grid_n;
};

// Store one output element (m, n) of sub-product g; returns the value that
// enters the Bz sum (0 otherwise).
template <typename T, int EPI>
__device__ __forceinline__ double epilogue(const GemmBatch<T> &batch, const GemmDesc<T> &g,
                                           int m, int n, T v)
{
    const int om = g.rmul * m + g.radd, on = g.cmul * n + g.cadd;
    if (EPI == EPI_STORE) {
        g.C[(int64_t)om * g.ldc + on] = v;
    } else if (EPI == EPI_SCALE) {
        g.C[(int64_t)om * g.ldc + on] = v * g.E[(int64_t)om * g.lde + on];
    } else {
        const FieldOut &o = batch.out[g.prob];
        const int64_t off = (int64_t)(om + o.row_off) * batch.grid_n + on + o.col_off;
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
            return dv;
        }
    }
    return 0.0;
}

template <int NT>
__device__ __forceinline__ void bz_reduce(double part, double *dst)
{
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    const int tid = threadIdx.x;
    if ((tid & 31) == 0) red[tid >> 5] = part;
    __syncthreads();
    if (tid < 32) {
        double s = tid < NT / 32 ? red[tid] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (tid == 0) atomicAdd(dst, s);
    }
}

// ---------------------------------------------------------------------------
// cp.async helpers (16-byte chunks, zero-filled past the valid bytes).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, int bytes)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n"
                 :: "r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" :: "n"(N) : "memory"); }

// ---------------------------------------------------------------------------
// FP64 products on the tensor cores: mma.sync.m8n8k4 .f64.  A warp owns a
// 32 x 32 tile (4 x 4 mma tiles); the CTA is WM x WN warps.  A and B tiles
// of depth 16 stream through an ST-stage cp.async pipeline in shared memory.
// Fragment layouts (PTX ISA, m8n8k4 f64): A row = lane/4, col = lane%4;
// B row = lane%4, col = lane/4; C row = lane/4, cols 2(lane%4) + {0,1}.
// Shared-memory row strides (20 and BN + 8 doubles) make both fragment loads
// conflict-free (two wavefronts for 256 bytes).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(c0), "+d"(c1) : "d"(a), "d"(b));
}

template <int WM, int WN, int ST>
struct DmmaCfg {
    static constexpr int BM = 32 * WM, BN = 32 * WN, BK = 16, NT = WM * WN * 32;
    static constexpr int AST = BK + 4, BST = BN + 8;
    static constexpr size_t smem = (size_t)ST * (BM * AST + BK * BST) * sizeof(double);
};

template <int WM, int WN, int ST, int EPI>
__global__ void __launch_bounds__(WM * WN * 32)
k_gemm_dmma(const __grid_constant__ GemmBatch<double> batch)
{
    using Cfg = DmmaCfg<WM, WN, ST>;
    constexpr int BM = Cfg::BM, BN = Cfg::BN, BK = Cfg::BK, NT = Cfg::NT;
    constexpr int AST = Cfg::AST, BST = Cfg::BST;
    extern __shared__ __align__(16) double dsm[];
    double *As = dsm;                       // [ST][BM][AST]
    double *Bs = dsm + ST * BM * AST;       // [ST][BK][BST]

    const GemmDesc<double> &g = batch.d[blockIdx.z];
    const int M = g.M, N = g.N, K = g.K;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    if (m0 >= M || n0 >= N) return;
    const double *__restrict__ A = g.A;
    const double *__restrict__ B = g.B;
    const int lda = g.lda, ldb = g.ldb;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp / WN, wn = warp % WN;

    auto issue = [&](int stage, int k0) {
        double *as = As + stage * BM * AST;
        double *bs = Bs + stage * BK * BST;
#pragma unroll
        for (int c = tid; c < BM * (BK / 2); c += NT) {
            const int r = c / (BK / 2), cc = c % (BK / 2);
            const int gm = m0 + r, gk = k0 + 2 * cc;
            int bytes = (gm < M) ? (K - gk) * 8 : 0;
            bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
            const double *src = bytes ? A + (int64_t)gm * lda + gk : A;
            cp_async16(as + r * AST + 2 * cc, src, bytes);
        }
#pragma unroll
        for (int c = tid; c < BK * (BN / 2); c += NT) {
            const int r = c / (BN / 2), cc = c % (BN / 2);
            const int gk = k0 + r, gn = n0 + 2 * cc;
            int bytes = (gk < K) ? (N - gn) * 8 : 0;
            bytes = bytes < 0 ? 0 : (bytes > 16 ? 16 : bytes);
            const double *src = bytes ? B + (int64_t)gk * ldb + gn : B;
            cp_async16(bs + r * BST + 2 * cc, src, bytes);
        }
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

    const int nk = (K + BK - 1) / BK;
#pragma unroll
    for (int s = 0; s < ST - 1; s++) {
        if (s < nk) issue(s, s * BK);
        cp_async_commit();
    }
    const int ar = wm * 32 + (lane >> 2), ac = lane & 3;
    const int br = lane & 3, bc = wn * 32 + (lane >> 2);
    for (int kt = 0; kt < nk; kt++) {
        cp_async_wait<ST - 2>();
        __syncthreads();
        const int nxt = kt + ST - 1;
        if (nxt < nk) issue(nxt % ST, nxt * BK);
        cp_async_commit();
        const double *as = As + (kt % ST) * BM * AST;
        const double *bs = Bs + (kt % ST) * BK * BST;
#pragma unroll
        for (int ks = 0; ks < BK / 4; ks++) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; i++) a[i] = as[(ar + 8 * i) * AST + ks * 4 + ac];
#pragma unroll
            for (int j = 0; j < 4; j++) b[j] = bs[(ks * 4 + br) * BST + bc + 8 * j];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
        }
    }
    cp_async_wait<0>();

    double part = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int gm = m0 + wm * 32 + 8 * i + (lane >> 2);
        if (gm >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
#pragma unroll
            for (int t = 0; t < 2; t++) {
                const int gn = n0 + wn * 32 + 8 * j + 2 * (lane & 3) + t;
                if (gn < N) part += epilogue<double, EPI>(batch, g, gm, gn, acc[i][j][t]);
            }
        }
    }
    if (EPI == EPI_FIELD && batch.out[g.prob].kind == 3) bz_reduce<NT>(part, batch.out[g.prob].bz_sum);
}

// ---------------------------------------------------------------------------
// FP32 products (mixed precision) on the FP32 cores: BM x BN per CTA,
// TM x TN outputs per thread, register-staged double buffering.
// ---------------------------------------------------------------------------
template <int BM, int BN, int BK, int TM, int TN, int EPI>
__global__ void __launch_bounds__((BM / TM) * (BN / TN))
k_gemm_f32(const __grid_constant__ GemmBatch<float> batch)
{
    constexpr int NT = (BM / TM) * (BN / TN);
    const GemmDesc<float> &g = batch.d[blockIdx.z];
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    if (m0 >= g.M || n0 >= g.N) return;
    __shared__ float As[2][BK][BM + 4];
    __shared__ float Bs[2][BK][BN];
    const int tid = threadIdx.x;
    const int tn = tid % (BN / TN), tm = tid / (BN / TN);
    float acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; i++)
#pragma unroll
        for (int j = 0; j < TN; j++) acc[i][j] = 0.f;
    constexpr int A_PER = (BM * BK + NT - 1) / NT, B_PER = (BK * BN + NT - 1) / NT;
    float ra[A_PER], rb[B_PER];
    auto load_regs = [&](int k0) {
#pragma unroll
        for (int r = 0; r < A_PER; r++) {
            const int e = tid + r * NT;
            const int mm = e / BK, kk = e % BK;
            const int gm = m0 + mm, gk = k0 + kk;
            ra[r] = (e < BM * BK && gm < g.M && gk < g.K) ? g.A[(int64_t)gm * g.lda + gk] : 0.f;
        }
#pragma unroll
        for (int r = 0; r < B_PER; r++) {
            const int e = tid + r * NT;
            const int kk = e / BN, nn = e % BN;
            const int gk = k0 + kk, gn = n0 + nn;
            rb[r] = (e < BK * BN && gk < g.K && gn < g.N) ? g.B[(int64_t)gk * g.ldb + gn] : 0.f;
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
            float a[TM], b[TN];
#pragma unroll
            for (int i = 0; i < TM; i++) a[i] = As[buf][kk][tm * TM + i];
#pragma unroll
            for (int j = 0; j < TN; j++) b[j] = Bs[buf][kk][tn + j * (BN / TN)];
#pragma unroll
            for (int i = 0; i < TM; i++)
#pragma unroll
                for (int j = 0; j < TN; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        if (kt + 1 < nk) store_smem(buf ^ 1);
        __syncthreads();
    }
    double part = 0;
#pragma unroll
    for (int i = 0; i < TM; i++) {
        const int gm = m0 + tm * TM + i;
        if (gm >= g.M) continue;
#pragma unroll
        for (int j = 0; j < TN; j++) {
            const int gn = n0 + tn + j * (BN / TN);
            if (gn < g.N) part += epilogue<float, EPI>(batch, g, gm, gn, acc[i][j]);
        }
    }
    if (EPI == EPI_FIELD && batch.out[g.prob].kind == 3) bz_reduce<NT>(part, batch.out[g.prob].bz_sum);
}

// ---------------------------------------------------------------------------
// Fold passes.  A natural R x C matrix (row stride ld2(C)) becomes
//   columns: U = [x_j + x_{C-1-j}]_{j<mid} ++ [x_mid]  (R x He, stride ld2(He))
//            V = [x_j - x_{C-1-j}]_{j<mid}             (R x Ho, stride ld2(Ho)),
//            V stored after U;
//   rows:    the same on rows; U rows 0..He-1 then V rows, stride ld2(C).
// ---------------------------------------------------------------------------
template <typename T>
struct FoldDesc {
    const T *src;
    T *dst;
    int R, C, by_rows;
};

template <typename T>
struct FoldBatch {
    FoldDesc<T> d[NPROB];
};

template <typename T>
__global__ void __launch_bounds__(256) k_fold(const __grid_constant__ FoldBatch<T> fb)
{
    // blockIdx.y: row, x: columns (grid-stride), z: problem
    const FoldDesc<T> &f = fb.d[blockIdx.z];
    const int R = f.R, C = f.C, ldc = ld2(C);
    for (int i = blockIdx.y; i < R; i += gridDim.y) {
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < C; j += gridDim.x * blockDim.x) {
            if (!f.by_rows) {
                const int he = (C + 1) / 2, mid = (C - 1) / 2;
                const T *row = f.src + (int64_t)i * ldc;
                if (j < he) {
                    f.dst[(int64_t)i * ld2(he) + j] = j < mid ? row[j] + row[C - 1 - j] : row[mid];
                } else {
                    const int jj = j - he;
                    T *V = f.dst + (int64_t)R * ld2(he);
                    V[(int64_t)i * ld2(C - he) + jj] = row[jj] - row[C - 1 - jj];
                }
            } else {
                const int he = (R + 1) / 2, mid = (R - 1) / 2;
                T v;
                if (i < he) {
                    v = i < mid ? f.src[(int64_t)i * ldc + j] + f.src[(int64_t)(R - 1 - i) * ldc + j]
                                : f.src[(int64_t)mid * ldc + j];
                } else {
                    const int ii = i - he;
                    v = f.src[(int64_t)ii * ldc + j] - f.src[(int64_t)(R - 1 - ii) * ldc + j];
                }
                f.dst[(int64_t)i * ldc + j] = v;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Right-hand sides (fields.py:112-230).  A CTA computes an 8 x 32 patch of
// nodes; the summed half-step densities and the full currents it
// differentiates are staged with a one-node halo in shared memory.  Outputs
// are natural matrices with row stride ld2(cols).
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
    int with_phi;
};

__device__ __forceinline__ double psum(const double *a, int np, int64_t plane, int64_t i)
{
    return np == 2 ? a[i] + a[i + plane] : a[i];
}

constexpr int RHS_TY = 8, RHS_TX = 32;

template <typename T>
__global__ void __launch_bounds__(RHS_TX * RHS_TY)
k_fields_rhs(RhsArgs a, T *X0, T *X1, T *X2, T *X3, T *X4, T *X5, T *X6)
{
    __shared__ double s_ro[RHS_TY + 2][RHS_TX + 2], s_jz[RHS_TY + 2][RHS_TX + 2];
    __shared__ double s_jx[RHS_TY + 2][RHS_TX + 2], s_jy[RHS_TY + 2][RHS_TX + 2];
    const int N = a.N, n = N - 2;
    const int ldN = ld2(N), ldn = ld2(n);
    const int64_t plane = (int64_t)N * N;
    const int i0 = blockIdx.y * RHS_TY - 1, j0 = blockIdx.x * RHS_TX - 1;
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && threadIdx.y == 0 && a.bz_sum)
        *a.bz_sum = 0.0;
    const int tid = threadIdx.y * RHS_TX + threadIdx.x;
    for (int e = tid; e < (RHS_TY + 2) * (RHS_TX + 2); e += RHS_TX * RHS_TY) {
        const int li = e / (RHS_TX + 2), lj = e % (RHS_TX + 2);
        const int gi = i0 + li, gj = j0 + lj;
        double ro = 0, jz = 0, jx = 0, jy = 0;
        if (gi >= 0 && gi < N && gj >= 0 && gj < N) {
            const int64_t q = (int64_t)gi * N + gj;
            const double rbf = a.rb_full[q] / a.rb_div, rbp = a.rb_prev[q] / a.rb_div;
            // (full + rho_beam_full + prev + rho_beam_prev) / 2, fields.py:194-197
            ro = (psum(a.ro_f, a.n_f, plane, q) + rbf + psum(a.ro_p, a.n_p, plane, q) + rbp) / 2;
            jz = (psum(a.jz_f, a.n_f, plane, q) + rbf + psum(a.jz_p, a.n_p, plane, q) + rbp) / 2;
            jx = psum(a.jx_f, a.n_f, plane, q);
            jy = psum(a.jy_f, a.n_f, plane, q);
        }
        s_ro[li][lj] = ro; s_jz[li][lj] = jz; s_jx[li][lj] = jx; s_jy[li][lj] = jy;
    }
    __syncthreads();
    const int li = threadIdx.y + 1, lj = threadIdx.x + 1;
    const int i = i0 + li, j = j0 + lj;
    if (i >= N || j >= N) return;
    const int64_t t = (int64_t)i * N + j;
    const bool inner = i >= 1 && i < N - 1 && j >= 1 && j < N - 1;
    const double h2 = a.h * 2;
    double dro_dx = 0, dro_dy = 0, djz_dx = 0, djz_dy = 0;
    if (inner) {
        dro_dx = (s_ro[li + 1][lj] - s_ro[li - 1][lj]) / h2;
        dro_dy = (s_ro[li][lj + 1] - s_ro[li][lj - 1]) / h2;
        djz_dx = (s_jz[li + 1][lj] - s_jz[li - 1][lj]) / h2;
        djz_dy = (s_jz[li][lj + 1] - s_jz[li][lj - 1]) / h2;
    }
    const double djx_dxi = (psum(a.jx_p, a.n_p, plane, t) - s_jx[li][lj]) / a.dxi;
    const double djy_dxi = (psum(a.jy_p, a.n_p, plane, t) - s_jy[li][lj]) / a.dxi;
    const double Ex_rhs = -(dro_dx - djx_dxi - a.c * a.Ex[t]);
    const double Ey_rhs = -(dro_dy - djy_dxi - a.c * a.Ey[t]);
    const double Bx_rhs = +(djz_dy - djy_dxi + a.c * a.Bx[t]);
    const double By_rhs = -(djz_dx - djx_dxi - a.c * a.By[t]);
    if (i >= 1 && i < N - 1) {
        const int64_t o = (int64_t)(i - 1) * ldN + j;
        X0[o] = (T)Ey_rhs;
        X1[o] = (T)Bx_rhs;
    }
    if (j >= 1 && j < N - 1) {
        const int64_t o = (int64_t)i * ldn + (j - 1);
        X2[o] = (T)Ex_rhs;
        X3[o] = (T)By_rhs;
    }
    double djx_dy = 0, djy_dx = 0;
    if (inner) {
        djx_dy = s_jx[li][lj + 1] - s_jx[li][lj - 1];
        djy_dx = s_jy[li + 1][lj] - s_jy[li - 1][lj];
    }
    X6[(int64_t)i * ldN + j] = (T)(-(djx_dy - djy_dx) / h2);
    if (inner) {
        const int64_t o = (int64_t)(i - 1) * ldn + (j - 1);
        const double djx_dx = s_jx[li + 1][lj] - s_jx[li - 1][lj];
        const double djy_dy = s_jy[li][lj + 1] - s_jy[li][lj - 1];
        X4[o] = (T)(-(djx_dx + djy_dy) / h2);
        if (a.with_phi)
            X5[o] = (T)(psum(a.ro_f, a.n_f, plane, t) - psum(a.jz_f, a.n_f, plane, t));
    }
}

// Bz mean removal and half average, plus the Dirichlet edges of the other
// planes (the reference pads its inner solutions with zeros).
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
        // Solutions vanish on their Dirichlet edges: Ex(0), By(4) on the first
        // and last column, Ey(1), Bx(3) on the first and last row, Ez(2),
        // Phi(6) on all four.  There the reference's combinations reduce to
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

// ---------------------------------------------------------------------------
// Workspace: two slots of N (N + 4) elements per problem (natural and folded
// matrices alternate between them), the raw Bz plane and its sum.
// ---------------------------------------------------------------------------
template <typename T>
struct Work {
    T *S1[NPROB], *S2[NPROB];
    double *bz_raw, *bz_sum;
};

static size_t slot_elems(int N) { return ((size_t)N * (N + 4) + 31) / 32 * 32; }

template <typename T>
static size_t work_bytes(int N)
{
    size_t b = 2 * NPROB * slot_elems(N) * sizeof(T);
    b = (b + 255) / 256 * 256;
    b += (size_t)N * N * sizeof(double);
    b = (b + 255) / 256 * 256;
    b += 256;
    return b;
}

template <typename T>
static Work<T> carve(void *ws, int N)
{
    Work<T> w;
    T *p = static_cast<T *>(ws);
    for (int i = 0; i < NPROB; i++) { w.S1[i] = p; p += slot_elems(N); }
    for (int i = 0; i < NPROB; i++) { w.S2[i] = p; p += slot_elems(N); }
    size_t off = 2 * NPROB * slot_elems(N) * sizeof(T);
    off = (off + 255) / 256 * 256;
    char *base = static_cast<char *>(ws);
    w.bz_raw = reinterpret_cast<double *>(base + off);
    off += (size_t)N * N * sizeof(double);
    off = (off + 255) / 256 * 256;
    w.bz_sum = reinterpret_cast<double *>(base + off);
    return w;
}

template <int WM, int WN, int ST, int EPI>
static int launch_dmma_cfg(const GemmBatch<double> &b, int nsub, int maxM, int maxN,
                           cudaStream_t st)
{
    using Cfg = DmmaCfg<WM, WN, ST>;
    static bool attr = false;
    if (!attr) {
        cudaError_t e = cudaFuncSetAttribute(k_gemm_dmma<WM, WN, ST, EPI>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)Cfg::smem);
        if (e != cudaSuccess) return cuda_check(e, "dmma smem attribute");
        attr = true;
    }
    dim3 grid((maxN + Cfg::BN - 1) / Cfg::BN, (maxM + Cfg::BM - 1) / Cfg::BM, nsub);
    k_gemm_dmma<WM, WN, ST, EPI><<<grid, Cfg::NT, Cfg::smem, st>>>(b);
    return LCB_OK;
}

template <int EPI>
static int launch_dmma(const GemmBatch<double> &b, int nsub, int maxM, int maxN, int N,
                       cudaStream_t st)
{
    if (N > 200) return launch_dmma_cfg<2, 2, 3, EPI>(b, nsub, maxM, maxN, st);
    return launch_dmma_cfg<1, 1, 3, EPI>(b, nsub, maxM, maxN, st);
}

template <int EPI>
static int launch_f32(const GemmBatch<float> &b, int nsub, int maxM, int maxN, int N,
                      cudaStream_t st)
{
    if (N > 200) {
        dim3 grid((maxN + 63) / 64, (maxM + 63) / 64, nsub);
        k_gemm_f32<64, 64, 16, 4, 4, EPI><<<grid, 256, 0, st>>>(b);
    } else {
        dim3 grid((maxN + 31) / 32, (maxM + 31) / 32, nsub);
        k_gemm_f32<32, 32, 16, 2, 2, EPI><<<grid, 256, 0, st>>>(b);
    }
    return LCB_OK;
}

static int launch_wave(const GemmBatch<double> &b, int nsub, int epi, int maxM, int maxN,
                       int N, cudaStream_t st)
{
    if (epi == EPI_STORE) return launch_dmma<EPI_STORE>(b, nsub, maxM, maxN, N, st);
    if (epi == EPI_SCALE) return launch_dmma<EPI_SCALE>(b, nsub, maxM, maxN, N, st);
    return launch_dmma<EPI_FIELD>(b, nsub, maxM, maxN, N, st);
}

static int launch_wave(const GemmBatch<float> &b, int nsub, int epi, int maxM, int maxN,
                       int N, cudaStream_t st)
{
    if (epi == EPI_STORE) return launch_f32<EPI_STORE>(b, nsub, maxM, maxN, N, st);
    if (epi == EPI_SCALE) return launch_f32<EPI_SCALE>(b, nsub, maxM, maxN, N, st);
    return launch_f32<EPI_FIELD>(b, nsub, maxM, maxN, N, st);
}

template <typename T>
static int run_wave(const GemmBatch<T> &b, int nsub, int epi, int N, cudaStream_t st,
                    const char *what)
{
    int maxM = 0, maxN = 0;
    for (int s = 0; s < nsub; s++) {
        maxM = b.d[s].M > maxM ? b.d[s].M : maxM;
        maxN = b.d[s].N > maxN ? b.d[s].N : maxN;
    }
    const int rc = launch_wave(b, nsub, epi, maxM, maxN, N, st);
    if (rc) return rc;
    LCB_LAUNCH_CHECK(what);
    return LCB_OK;
}

template <typename T>
static int run_fold(T *const *src, T *const *dst, const int *probs, int np, const int *rows,
                    const int *cols, int by_rows, int N, cudaStream_t st)
{
    FoldBatch<T> fb;
    memset(&fb, 0, sizeof(fb));
    for (int q = 0; q < np; q++) {
        const int p = probs[q];
        fb.d[q].src = src[p];
        fb.d[q].dst = dst[p];
        fb.d[q].R = rows[p];
        fb.d[q].C = cols[p];
        fb.d[q].by_rows = by_rows;
    }
    dim3 grid((unsigned)((N + 255) / 256), (unsigned)N, np);
    k_fold<T><<<grid, 256, 0, st>>>(fb);
    LCB_LAUNCH_CHECK("k_fold");
    return LCB_OK;
}

template <typename T>
static int solve(const lcb_compute_fields_args *a, const T *ops, cudaStream_t st)
{
    const int N = a->grid_steps, n = N - 2;
    const OpLayout L = op_layout(N);
    Work<T> w = carve<T>(a->workspace, N);
    // Phi (problem 5) is skipped when neither of its outputs is wanted.
    const bool with_phi = a->out_half.f[6] || a->out_full.f[6];

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
    r.with_phi = with_phi;
    {
        dim3 grid((N + RHS_TX - 1) / RHS_TX, (N + RHS_TY - 1) / RHS_TY);
        k_fields_rhs<T><<<grid, dim3(RHS_TX, RHS_TY), 0, st>>>(
            r, w.S1[0], w.S1[1], w.S1[2], w.S1[3], w.S1[4], w.S1[5], w.S1[6]);
        LCB_LAUNCH_CHECK("k_fields_rhs");
    }

    // Per problem: rows x cols of X; the left operator (S or C) acts along
    // the rows, the right operator along the columns; spectral matrix.
    const int rows[NPROB] = {n, n, N, N, n, n, N};
    const int cols[NPROB] = {N, N, n, n, n, n, N};
    const bool leftS[NPROB] = {true, true, false, false, true, true, false};
    const bool rightS[NPROB] = {false, false, true, true, true, true, false};
    const int mat[NPROB] = {OP_MX, OP_MX, OP_MXT, OP_MXT, OP_D, OP_D, OP_NM};
    auto op = [&](int id) { return ops + L.off[id]; };

    int probs[NPROB], np = 0;
    for (int p = 0; p < NPROB; p++)
        if (p != P_PHI || with_phi) probs[np++] = p;

    GemmBatch<T> b;
    memset(&b, 0, sizeof(b));
    b.grid_n = N;
    // right waves: S1 (natural) -> fold columns -> S2; S1 = S2 [U|V] * [TeT;ToT]
    auto right_wave = [&]() {
        int s = 0;
        for (int q = 0; q < np; q++) {
            const int p = probs[q];
            const int C = cols[p], he = (C + 1) / 2, ho = (C - 1) / 2;
            for (int par = 0; par < 2; par++, s++) {
                GemmDesc<T> &d = b.d[s];
                memset(&d, 0, sizeof(d));
                d.A = par ? w.S2[p] + (int64_t)rows[p] * ld2(he) : w.S2[p];
                d.lda = par ? ld2(ho) : ld2(he);
                const int id = rightS[p] ? (par ? OP_SOT : OP_SET) : (par ? OP_COT : OP_CET);
                d.B = op(id); d.ldb = (int)L.ld[id];
                d.M = rows[p]; d.K = par ? ho : he; d.N = par ? ho : he;
                d.rmul = 1; d.radd = 0; d.cmul = 2; d.cadd = par;
                d.C = w.S1[p]; d.ldc = ld2(C); d.prob = p;
            }
        }
        return s;
    };
    // left waves: S1 -> fold rows -> S2; out = [Te;To] [U;V] (rows interleaved)
    auto left_wave = [&](bool to_fields) {
        int s = 0;
        for (int q = 0; q < np; q++) {
            const int p = probs[q];
            const int R = rows[p], he = (R + 1) / 2, ho = (R - 1) / 2;
            for (int par = 0; par < 2; par++, s++) {
                GemmDesc<T> &d = b.d[s];
                memset(&d, 0, sizeof(d));
                const int id = leftS[p] ? (par ? OP_SO : OP_SE) : (par ? OP_CO : OP_CE);
                d.A = op(id); d.lda = (int)L.ld[id];
                d.B = w.S2[p] + (par ? (int64_t)he * ld2(cols[p]) : 0); d.ldb = ld2(cols[p]);
                d.M = par ? ho : he; d.K = par ? ho : he; d.N = cols[p];
                d.rmul = 2; d.radd = par; d.cmul = 1; d.cadd = 0;
                if (!to_fields) { d.C = w.S1[p]; d.ldc = ld2(cols[p]); }
                d.E = op(mat[p]); d.lde = (int)L.ld[mat[p]];
                d.prob = p;
            }
        }
        return s;
    };

    int rc;
    // wave 1: S1 = S1 R
    if ((rc = run_fold<T>(w.S1, w.S2, probs, np, rows, cols, 0, N, st))) return rc;
    if ((rc = run_wave<T>(b, right_wave(), EPI_STORE, N, st, "wave1"))) return rc;
    // wave 2: S1 = (L S1) o Mat
    if ((rc = run_fold<T>(w.S1, w.S2, probs, np, rows, cols, 1, N, st))) return rc;
    if ((rc = run_wave<T>(b, left_wave(false), EPI_SCALE, N, st, "wave2"))) return rc;
    // wave 3: S1 = S1 R
    if ((rc = run_fold<T>(w.S1, w.S2, probs, np, rows, cols, 0, N, st))) return rc;
    if ((rc = run_wave<T>(b, right_wave(), EPI_STORE, N, st, "wave3"))) return rc;
    // wave 4: fields = L S1
    if ((rc = run_fold<T>(w.S1, w.S2, probs, np, rows, cols, 1, N, st))) return rc;
    const int nsub = left_wave(true);
    // field index in lcb_fields: Ex 0, Ey 1, Ez 2, Bx 3, By 4, Bz 5, Phi 6
    const int fidx[NPROB] = {1, 3, 0, 4, 2, 6, 5};
    const int roff[NPROB] = {1, 1, 0, 0, 1, 1, 0};
    const int coff[NPROB] = {0, 0, 1, 1, 1, 1, 0};
    const int kind[NPROB] = {0, 0, 0, 0, 1, 2, 3};
    for (int p = 0; p < NPROB; p++) {
        FieldOut &o = b.out[p];
        const int f = fidx[p];
        o.half = a->out_half.f[f]; o.full = a->out_full.f[f];
        o.prev = a->fields_prev.f[f];
        o.row_off = roff[p]; o.col_off = coff[p]; o.kind = kind[p];
        o.bz_raw = w.bz_raw; o.bz_sum = w.bz_sum;
    }
    if ((rc = run_wave<T>(b, nsub, EPI_FIELD, N, st, "wave4"))) return rc;

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
        const int blocks = (int)((tot + 255) / 256);
        k_fields_finish<<<blocks, 256, 0, st>>>(fa);
        LCB_LAUNCH_CHECK("k_fields_finish");
    }
    return LCB_OK;
}

}  // namespace lcb

using namespace lcb;

extern "C" size_t lcb_field_operators_bytes(int grid_steps, int precision)
{
    if (grid_steps < 5 || (grid_steps % 2) == 0) return 0;
    const size_t el = precision == LCB_PREC_MIXED ? sizeof(float) : sizeof(double);
    return (size_t)op_layout(grid_steps).off[OP_COUNT] * el;
}

extern "C" int lcb_field_operators_build(int grid_steps, double h, double subtraction_coeff,
                                         int precision, void *operators, size_t bytes,
                                         void *stream)
{
    const int N = grid_steps;
    LCB_REQUIRE(N >= 5 && (N % 2) == 1, "grid_steps must be odd and >= 5 (got %d)", N);
    LCB_REQUIRE(precision == LCB_PREC_FP64 || precision == LCB_PREC_MIXED, "bad precision");
    LCB_REQUIRE(operators && bytes >= lcb_field_operators_bytes(N, precision),
                "operator buffer too small (%zu < %zu)", bytes,
                lcb_field_operators_bytes(N, precision));
    LCB_REQUIRE(((uintptr_t)operators & 255) == 0, "operator buffer must be 256-byte aligned");
    LCB_REQUIRE(h > 0, "transverse step must be > 0");
    const OpLayout L = op_layout(N);
    const int blocks = (int)((L.off[OP_COUNT] + 255) / 256);
    if (precision == LCB_PREC_MIXED)
        k_build_ops<float><<<blocks, 256, 0, as_stream(stream)>>>(
            N, h, subtraction_coeff, L, static_cast<float *>(operators));
    else
        k_build_ops<double><<<blocks, 256, 0, as_stream(stream)>>>(
            N, h, subtraction_coeff, L, static_cast<double *>(operators));
    LCB_LAUNCH_CHECK("k_build_ops");
    return LCB_OK;
}

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
    LCB_REQUIRE(a->operators && ((uintptr_t)a->operators & 255) == 0,
                "operators must be a 256-byte aligned buffer from lcb_field_operators_build");
    LCB_REQUIRE(a->currents_full.n_planes >= 1 && a->currents_full.n_planes <= 2 &&
                a->currents_prev.n_planes >= 1 && a->currents_prev.n_planes <= 2,
                "currents must have 1 or 2 planes");
    LCB_REQUIRE(a->rho_beam_divisor != 0.0, "rho_beam_divisor is 0");
    for (int f : {0, 1, 3, 4}) LCB_REQUIRE(a->fields.f[f], "fields plane %d is NULL", f);
    for (int f = 0; f < 6; f++) LCB_REQUIRE(a->fields_prev.f[f], "fields_prev plane %d is NULL", f);
    cudaStream_t st = as_stream(stream);
    if (a->precision == LCB_PREC_MIXED)
        return solve<float>(a, static_cast<const float *>(a->operators), st);
    LCB_REQUIRE(a->precision == LCB_PREC_FP64, "bad precision %d", a->precision);
    return solve<double>(a, static_cast<const double *>(a->operators), st);
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
                "allocation-free entry point has %zu (largest grid: 261 in FP64, "
                "359 in mixed precision) -- use lcb_compute_fields with a workspace",
                a->grid_steps, a->precision, need, (size_t)LCB_NOALLOC_FIELDS_SCRATCH_BYTES);
    void *scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    lcb_compute_fields_args b = *a;
    b.workspace = scratch;
    b.workspace_bytes = LCB_NOALLOC_FIELDS_SCRATCH_BYTES;
    return lcb_compute_fields(&b, stream);
}
