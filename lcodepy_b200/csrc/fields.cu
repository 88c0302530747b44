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
// All products run on the int8 tensor cores (tcgen05) on sliced operands,
// exactly: eight slices reproduce FP64 accuracy, four FP32 accuracy (mixed
// precision).
#include <cstdlib>
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

// Leading dimension of the natural-layout matrices (right-hand sides,
// products): padded to an even number of elements.
__host__ __device__ constexpr int ld2(int c) { return (c + 1) & ~1; }

// Operands of the tensor-core transforms are written as int8 slices,
//     x = 2^E (s_0 2^-6 + s_1 2^-13 + ... + s_{NS-1} 2^-(6 + 7 (NS - 1))),
// |s_i| <= 64: four slices for FP32 operands (mixed precision), eight for
// FP64 ones.  slices_of returns the slices of x * scale (|x * scale| <= 1),
// each as a byte in the low bits: the sum with 1.5 * 2^23 (FP32) or
// 1.5 * 2^52 (FP64) rounds to an integer held in the low mantissa bits.
template <int NS>
__device__ __forceinline__ void slices_of(double x, double scale, unsigned sl[NS]);

template <>
__device__ __forceinline__ void slices_of<4>(double x, double scale, unsigned sl[4])
{
    const float MG = 12582912.0f;
    float u = (float)x * (float)scale * 64.f;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float v = u + MG;
        sl[i] = __float_as_uint(v) & 0xFFu;
        u = (u - (v - MG)) * 128.f;
    }
}

template <>
__device__ __forceinline__ void slices_of<8>(double x, double scale, unsigned sl[8])
{
    const double MG = 6755399441055744.0;
    double u = x * scale * 64.0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const double v = u + MG;
        sl[i] = (unsigned)__double_as_longlong(v) & 0xFFu;
        u = (u - (v - MG)) * 128.0;
    }
}

// The data operands' slices come from one float-to-integer conversion:
// X = round(x * scale * 2^(6 + 7 (NS - 1))), the value x * scale rounded to
// the last slice's unit as slices_of rounds it.  Its balanced base-128
// digits (|s| <= 64, the top one may reach 64) are the unsigned 7-bit fields
// of B = X + 64 (1 + 2^7 + ... + 2^(7 (NS - 1))) less 64 each; the fields
// are returned with the 64 still added (0 .. 128), and put_slices4 removes
// it from four packed bytes at once.
__device__ __forceinline__ void slices_biased(double x, double scale, unsigned sl[8])
{
    const long long X = __double2ll_rn(x * scale * 36028797018963968.0);   // 2^55
    const unsigned long long B = (unsigned long long)X + 0x81020408102040ull;
    const unsigned lo = (unsigned)B, hi = (unsigned)(B >> 32);
    sl[7] = lo & 127u;
    sl[6] = (lo >> 7) & 127u;
    sl[5] = (lo >> 14) & 127u;
    sl[4] = (lo >> 21) & 127u;
    sl[3] = __funnelshift_r(lo, hi, 28) & 127u;
    sl[2] = (hi >> 3) & 127u;
    sl[1] = (hi >> 10) & 127u;
    sl[0] = hi >> 17;
}
__device__ __forceinline__ void slices_biased(float x, double scale, unsigned sl[4])
{
    const int X = __float2int_rn(x * (float)scale * 134217728.0f);          // 2^27
    const unsigned B = (unsigned)X + 0x8102040u;
    sl[3] = B & 127u;
    sl[2] = (B >> 7) & 127u;
    sl[1] = (B >> 14) & 127u;
    sl[0] = B >> 21;
}

// Slices per element of an operand of type T (one byte each: the sliced
// form takes the same storage as T).
template <typename T> struct Slices { static constexpr int n = (int)sizeof(T); };

// A float upper bound of |x| (rounded up), for the per-problem maxima.
__device__ __forceinline__ float abs_bound(float x) { return fabsf(x); }
__device__ __forceinline__ float abs_bound(double x) { return __double2float_ru(fabs(x)); }

// Exponent E with m <= 2^E for m >= 0 (0 for m = 0).
__device__ __forceinline__ int bound_exp(float m)
{
    if (!(m > 0.f)) return 0;
    int e;
    frexpf(m, &e);
    return e;
}


struct OpLayout {
    int64_t off[OP_COUNT + 1];  // element offsets, 32-element aligned
    int64_t rows[OP_COUNT], cols[OP_COUNT], ld[OP_COUNT];
};


// ---------------------------------------------------------------------------
// Operand storage: NS int8 slices per element (four for mixed precision,
// eight for FP64), cut into the tiles the tensor-core GEMM streams (zero
// padded), each tile stored in the tensor cores' no-swizzle core-matrix
// order, and the NS slices of a tile back to back, so that one contiguous
// bulk copy fills a shared-memory stage.
//   A role (M x K, K-major): 128 x 32 tiles of 4096 bytes per slice, slice i
//     of tile (mt, kt) at ((mt KT + kt) NS + i) 4096, element (r, k) at
//     (r/8) 256 + (k/16) 128 + (r%8) 16 + k%16;
//   B role (K x N, N-major): 32 x 64 tiles of 2048 bytes per slice, slice i
//     of tile (kt, nt) at ((nt KT + kt) NS + i) 2048, element (k, n) at
//     (n/16) 512 + (k/8) 128 + (k%8) 16 + n%16.
// ---------------------------------------------------------------------------
constexpr int TL_M = 128, TL_K = 32, TL_N = 64;
__host__ __device__ constexpr int ntiles(int x, int t) { return (x + t - 1) / t; }
__host__ __device__ constexpr int64_t a_plane_bytes(int M, int K)
{
    return (int64_t)ntiles(M, TL_M) * ntiles(K, TL_K) * (TL_M * TL_K);
}
__host__ __device__ constexpr int64_t b_plane_bytes(int K, int N)
{
    return (int64_t)ntiles(K, TL_K) * ntiles(N, TL_N) * (TL_K * TL_N);
}
// Offset of slice i of element (r, k) (A role) or (k, n) (B role): the NS
// slices of one tile are stored back to back, so that a stage of the
// tensor-core pipeline is one contiguous copy per operand.
__host__ __device__ inline int64_t a_tile_off(int r, int k, int KT, int NS, int i)
{
    return ((((int64_t)(r >> 7) * KT + (k >> 5)) * NS + i) << 12) + ((r & 127) >> 3) * 256 +
           ((k & 31) >> 4) * 128 + (r & 7) * 16 + (k & 15);
}
__host__ __device__ inline int64_t b_tile_off(int k, int n, int KT, int NS, int i)
{
    return ((((int64_t)(n >> 6) * KT + (k >> 5)) * NS + i) << 11) + ((n & 63) >> 4) * 512 +
           ((k & 31) >> 3) * 128 + (k & 7) * 16 + (n & 15);
}

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
        L.ld[i] = c[i];
        // transform blocks: sizeof(T) tiled slice planes (as many elements of
        // T as one plane has bytes), A role for the left operators (SE SO CE
        // CO), B role for the right ones (transposed); spectral matrices in T
        const bool a_role = i == OP_SE || i == OP_SO || i == OP_CE || i == OP_CO;
        const int64_t words = i < OP_D
            ? (a_role ? a_plane_bytes((int)r[i], (int)c[i]) : b_plane_bytes((int)r[i], (int)c[i]))
            : r[i] * L.ld[i];
        o += (words + 31) / 32 * 32;
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

// The transform blocks as NS tiled int8 slice planes (bound 2); the thread
// of padded element e writes its NS slices.
template <int NS>
__global__ void k_build_slices(int N, OpLayout L, uint8_t *bytes)
{
    const int n = N - 2;
    for (int b = 0; b < OP_D; b++) {
        const bool a_role = b == OP_SE || b == OP_SO || b == OP_CE || b == OP_CO;
        const int R = (int)L.rows[b], C = (int)L.cols[b];
        // padded extents: A role 128-row x 32-col tiles, B role 32 x 64
        const int Rp = a_role ? ntiles(R, TL_M) * TL_M : ntiles(R, TL_K) * TL_K;
        const int Cp = a_role ? ntiles(C, TL_K) * TL_K : ntiles(C, TL_N) * TL_N;
        const int KT = a_role ? ntiles(C, TL_K) : ntiles(R, TL_K);
        uint8_t *base = bytes + (int64_t)NS * L.off[b];
        for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)Rp * Cp;
             e += (int64_t)gridDim.x * blockDim.x) {
            const int r = (int)(e / Cp), q = (int)(e % Cp);
            double v = 0;
            if (r < R && q < C) {
                switch (b) {
                case OP_SE: v = dst1(2 * r, q, n); break;
                case OP_SO: v = dst1(2 * r + 1, q, n); break;
                case OP_SET: v = dst1(2 * q, r, n); break;
                case OP_SOT: v = dst1(2 * q + 1, r, n); break;
                case OP_CE: v = dct1(2 * r, q, N); break;
                case OP_CO: v = dct1(2 * r + 1, q, N); break;
                case OP_CET: v = dct1(2 * q, r, N); break;
                case OP_COT: v = dct1(2 * q + 1, r, N); break;
                }
            }
            unsigned sl[NS];
            slices_of<NS>(v, 0.5, sl);
#pragma unroll
            for (int i = 0; i < NS; i++)
                base[a_role ? a_tile_off(r, q, KT, NS, i) : b_tile_off(r, q, KT, NS, i)] = (uint8_t)sl[i];
        }
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
    // mixed precision: max |element| of a data operand (float bits, written
    // by the fold pass that produced it); NULL for a transform block, whose
    // elements are bounded by 2
    const unsigned *amax_a, *amax_b;
    // which operand is a transform block (1: A, 2: B), whose copies may be
    // issued before the predecessor kernel has finished
    int const_op;
};

enum Epi { EPI_STORE = 0, EPI_SCALE = 1, EPI_FIELD = 2 };

// The fields of a product that its epilogue reads, held in registers.
template <typename T>
struct EpiDesc {
    T *C; const T *E;
    int ldc, lde, rmul, radd, cmul, cadd, M, N;
};

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
    int nsub;             // products in d (the persistent wave walks their tiles)
    unsigned *amax_out;   // mixed: per-problem max |stored value| (zeroed), or NULL
};

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
// The dense transforms on the 5th-generation tensor cores, exact in integer
// arithmetic.  Every operand element is written as NS int8 slices,
//     x = 2^E (s_0 2^-6 + s_1 2^-13 + ... ),  |s_i| <= 64,
// with E the exponent of its matrix's bound (the producer of the matrix
// records its largest element; a fold at most doubles it; transform blocks
// are bounded by 2): NS = 4 for FP32 operands (mixed precision,
// representation error below 2^(E-28)) and NS = 8 for FP64 ones (below
// 2^(E-56)).  The product of two such matrices is the sum over slice pairs
// (i, j) of int8 GEMMs scaled by 2^-(12 + 7(i+j)); the pairs with
// i + j < NS go to NS int32 accumulators in tensor memory (one per i + j),
// where tcgen05.mma kind::i8 sums them exactly (|sum| < NS 64^2 K < 2^31
// for these K).  The epilogue combines them in 64-bit integers: the result
// is as accurate as a product in the operands' precision and, unlike
// floating-point tensor-core accumulation, free of rounding bias and
// independent of summation order.
//
// CTA: 256 threads; a 128 x 64 output tile in tensor memory (64 columns per
// accumulator), K in stages of 32.  The operands are stored pre-tiled (see
// the tile geometry above), so a stage is 2 NS bulk copies issued by one
// lane of warp 0, completing on the stage's mbarrier; the same lane issues
// the MMAs and commits them to a second mbarrier per stage, which gates the
// refill of that stage's buffers.  A final one-shot commit releases the
// epilogue: all eight warps read TMEM (warp w: lanes 32 (w % 4), columns
// 32 (w / 4)) and store through shared memory.
// ---------------------------------------------------------------------------
constexpr int I8_BM = 128, I8_BK = 32;
constexpr int I8_A_SLICE = I8_BM * I8_BK;            // bytes per slice of the A tile

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

// 64-bit shared-memory matrix descriptor, no swizzle (start, LBO, SBO in bytes).
__device__ __forceinline__ uint64_t umma_desc(unsigned addr, unsigned lbo, unsigned sbo)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ull << 46);
}

// Instruction descriptor: kind::i8, s32 accumulator, signed int8 A (K-major)
// and B (MN-major), M = 128, N = BN.
template <int BN>
__device__ __forceinline__ unsigned i8_idesc()
{
    return (2u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((unsigned)(BN >> 3) << 17) |
           ((unsigned)(I8_BM >> 4) << 24);
}

// Exponent of an operand's bound: a data operand's recorded maximum, or 2
// for a transform block.
__device__ __forceinline__ int operand_exp(const unsigned *amax)
{
    // a fold output is bounded by twice its source's largest element
    return amax ? bound_exp(2.f * __uint_as_float(*amax)) : 1;
}

__device__ __forceinline__ bool mbar_wait(unsigned mbar, unsigned parity)
{
    // bounded: a phase that never completes ends the wait after ~2^22 polls
    for (int it = 0; it < (1 << 22); it++) {
        unsigned done;
        asm volatile("{\n.reg .pred P1;\nmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n"
                     "selp.b32 %0, 1, 0, P1;\n}\n"
                     : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// Epilogue of the integer products, split so that a group of outputs can
// load what it needs (scale factor, previous field) before storing.
template <int EPI, typename T, typename G>
__device__ __forceinline__ double epi_pre(const FieldOut &o, int grid_n, const G &g, int m, int n)
{
    const int om = g.rmul * m + g.radd, on = g.cmul * n + g.cadd;
    if (EPI == EPI_SCALE) return (double)g.E[(int64_t)om * g.lde + on];
    if (EPI == EPI_FIELD) {
        if ((o.kind == 0 && o.full) || (o.kind == 1 && o.half))
            return o.prev[(int64_t)(om + o.row_off) * grid_n + on + o.col_off];
    }
    return 0.0;
}

template <int EPI, typename T, typename G>
__device__ __forceinline__ double epi_apply(const FieldOut &o, int grid_n, const G &g, int m, int n,
                                            T v, double pre, float &vmax)
{
    const int om = g.rmul * m + g.radd, on = g.cmul * n + g.cadd;
    if (EPI == EPI_STORE) {
        g.C[(int64_t)om * g.ldc + on] = v;
        vmax = fmaxf(vmax, abs_bound(v));
    } else if (EPI == EPI_SCALE) {
        const T st = v * (T)pre;
        g.C[(int64_t)om * g.ldc + on] = st;
        vmax = fmaxf(vmax, abs_bound(st));
    } else {
        const int64_t off = (int64_t)(om + o.row_off) * grid_n + on + o.col_off;
        const double dv = (double)v;
        if (o.kind == 0) {
            if (o.half) o.half[off] = dv;
            if (o.full) o.full[off] = 2 * dv - pre;
        } else if (o.kind == 1) {
            if (o.full) o.full[off] = dv;
            if (o.half) o.half[off] = (dv + pre) / 2;
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

template <int NS, int BN>
struct I8Cfg {
    // a CTA covers BN columns: two consecutive 64-wide B tiles (BN = 128,
    // one CTA per SM, all of tensor memory), a whole one (BN = 64, two CTAs
    // per SM) or, for BN = 32, the contiguous half of one (its N core-matrix
    // groups 0-1 or 2-3)
    static_assert((TL_N % BN == 0 || BN == 2 * TL_N) && BN % 16 == 0, "tile width");
    static constexpr int B_SLICE = I8_BK * BN;                         // bytes
    static constexpr int STAGE = NS * (I8_A_SLICE + B_SLICE);          // bytes
    static constexpr int ST = BN > TL_N ? 6 : (4 * STAGE <= 100 * 1024 ? 4 : 2);  // pipeline stages
    static constexpr int TMEM_COLS = NS * BN;                          // power of two
    static constexpr int THREADS = BN > TL_N ? 512 : 256;              // 16 or 8 warps
    static constexpr int CW = BN / (THREADS / 128);                    // epilogue columns per warp
    static constexpr size_t smem = (size_t)ST * STAGE + 128;   // + 2 ST + 1 barriers, TMEM slot
};

__device__ __forceinline__ void bulk_g2s(unsigned dst, const void *src, unsigned bytes, unsigned mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
                 :: "r"(dst), "l"(src), "r"(bytes), "r"(mbar) : "memory");
}

template <typename T, int BN, int EPI>
__global__ void __launch_bounds__(I8Cfg<Slices<T>::n, BN>::THREADS, 512 / I8Cfg<Slices<T>::n, BN>::TMEM_COLS)
k_gemm_i8(const __grid_constant__ GemmBatch<T> batch)
{
    constexpr int NS = Slices<T>::n;
    using Cfg = I8Cfg<NS, BN>;
    constexpr int ST = Cfg::ST;
    constexpr int CW = Cfg::CW;           // epilogue columns per warp
    static_assert(Cfg::TMEM_COLS == 256 || Cfg::TMEM_COLS == 512, "tensor memory columns");
    static_assert(Cfg::THREADS / 32 * 32 * (CW + 1) * sizeof(T) <= (size_t)ST * Cfg::STAGE,
                  "epilogue staging");
    extern __shared__ __align__(1024) uint8_t i8sm[];
    uint64_t *full = reinterpret_cast<uint64_t *>(i8sm + ST * Cfg::STAGE);   // [ST] copies landed
    uint64_t *done = full + ST;                                             // [ST] MMAs finished
    uint64_t *fin = done + ST;                                              // all MMAs finished
    unsigned *tslot = reinterpret_cast<unsigned *>(fin + 1);

    const GemmDesc<T> &g = batch.d[blockIdx.z];
    // register copies of what the epilogue reads (parameter reads indexed by
    // blockIdx.z are slow)
    EpiDesc<T> ge;
    ge.C = g.C; ge.E = g.E; ge.ldc = g.ldc; ge.lde = g.lde; ge.rmul = g.rmul; ge.radd = g.radd;
    ge.cmul = g.cmul; ge.cadd = g.cadd; ge.M = g.M; ge.N = g.N;
    const FieldOut go = batch.out[g.prob];
    const int grid_n = batch.grid_n;
    const int M = g.M, N = g.N, K = g.K;
    const int m0 = blockIdx.y * I8_BM, n0 = blockIdx.x * BN;
    if (m0 >= M || n0 >= N) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int KT = ntiles(K, TL_K);
    // this CTA's tile rows of A and tile column of B (NS slices per tile)
    const uint8_t *At = reinterpret_cast<const uint8_t *>(g.A) + (int64_t)blockIdx.y * KT * NS * I8_A_SLICE;
    const uint8_t *Bt = reinterpret_cast<const uint8_t *>(g.B) + (int64_t)(n0 / TL_N) * KT * NS * (TL_K * TL_N) +
                        ((n0 % TL_N) >> 4) * 512;
    // BN = 128: the second B tile column (or the first again past the last
    // one; its products land in columns that are never stored)
    const uint8_t *Bt2 = (n0 / TL_N + 1) < ntiles(N, TL_N) ? Bt + (int64_t)KT * NS * (TL_K * TL_N) : Bt;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tslot)), "r"(Cfg::TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0)
        for (int q = 0; q < 2 * ST + 1; q++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(full + q)), "r"(1)
                         : "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tslot;
    const unsigned idesc = i8_idesc<BN>();

    // Stage copies (lane 0 of warp 0): part 1 = A slices, part 2 = B slices,
    // part 3 = both; the stage's barrier expects all of its bytes once.
    auto load = [&](int kt, int part, bool expect) {
        if (warp != 0 || lane != 0) return;
        const int buf = kt % ST;
        const unsigned sA = smem_u32(i8sm + buf * Cfg::STAGE);
        const unsigned sB = sA + NS * I8_A_SLICE;
        const unsigned mb = smem_u32(full + buf);
        if (expect)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;"
                         :: "r"((unsigned)Cfg::STAGE), "r"(mb) : "memory");
#pragma unroll
        for (int i = 0; i < NS; i++) {
            if (part & 1)
                bulk_g2s(sA + i * I8_A_SLICE, At + ((int64_t)kt * NS + i) * I8_A_SLICE, I8_A_SLICE, mb);
            if (part & 2) {
                if constexpr (BN > TL_N) {
                    constexpr int HB = TL_K * TL_N;   // one 64-wide tile slice
                    bulk_g2s(sB + i * Cfg::B_SLICE, Bt + ((int64_t)kt * NS + i) * HB, HB, mb);
                    bulk_g2s(sB + i * Cfg::B_SLICE + HB, Bt2 + ((int64_t)kt * NS + i) * HB, HB, mb);
                } else {
                    bulk_g2s(sB + i * Cfg::B_SLICE, Bt + ((int64_t)kt * NS + i) * (TL_K * TL_N),
                             Cfg::B_SLICE, mb);
                }
            }
        }
    };
    // the first stages' transform-block copies go out before the wait: the
    // blocks are written once, when the operators are built
    const int npre = ST < KT ? ST : KT;
    const int cpart = g.const_op, dpart = 3 - cpart;
    if (cpart)
        for (int kt = 0; kt < npre; kt++) load(kt, cpart, true);
    // the prologue above overlaps the predecessor's tail (programmatic launch)
    pdl_wait();
    pdl_trigger();
    for (int kt = 0; kt < npre; kt++) load(kt, cpart ? dpart : 3, !cpart);
    const int ea = operand_exp(g.amax_a), eb = operand_exp(g.amax_b);

    // epilogue layout: warp w stores TMEM lanes 32 (w % 4) .. + 31 (tile rows)
    // and columns CW (w / 4) .. + CW - 1; pass `it` of a lane covers element
    // it * 32 + lane of the warp's 32 x CW block (lanes along a row).  The
    // values the epilogue reads (spectral factors, previous fields) are
    // loaded here, so that their latency hides behind the main loop.
    const int rq = warp & 3, ch = warp >> 2;
    double pre[CW];
#pragma unroll
    for (int it = 0; it < CW; it++) {
        const int e = it * 32 + lane, row = e / CW, col = e % CW;
        const int gm = m0 + 32 * rq + row, gn = n0 + CW * ch + col;
        pre[it] = (EPI != EPI_STORE && gm < M && gn < N)
                      ? epi_pre<EPI, T>(go, grid_n, ge, gm, gn) : 0.0;
    }

    bool ok = true;
    if (warp == 0) {
        // warp 0 streams the stages (eight bulk copies each: four A and four
        // B slice tiles) and issues the MMAs from lane 0; the whole warp
        // follows the loop so that lane 0 never diverges from idle lanes
        for (int kt = 0; kt < KT; kt++) {
            const int buf = kt % ST;
            ok &= mbar_wait(smem_u32(full + buf), (kt / ST) & 1);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned a0 = smem_u32(i8sm + buf * Cfg::STAGE);
            const unsigned b0 = a0 + NS * I8_A_SLICE;
            if (lane == 0) {
#pragma unroll
            for (int i = 0; i < NS; i++) {
#pragma unroll
                for (int j = 0; j < NS - i; j++) {
                    const uint64_t da = umma_desc(a0 + i * I8_A_SLICE, 128, 256);
                    const uint64_t db = umma_desc(b0 + j * Cfg::B_SLICE, 128, 512);
                    const unsigned acc = tmem + (unsigned)((i + j) * BN);
                    const unsigned en = (kt > 0 || i > 0) ? 1u : 0u;
                    asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, "
                                 "{%5, %5, %5, %5}, p;\n}\n"
                                 :: "r"(acc), "l"(da), "l"(db), "r"(idesc), "r"(en), "r"(0u)
                                 : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_u32(done + buf)) : "memory");
            if (kt == KT - 1)
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             :: "r"(smem_u32(fin)) : "memory");
            }
            __syncwarp();
            // refill the buffer of stage kt - 1 (its MMAs were issued a stage ago)
            const int nxt = kt - 1 + ST;
            if (kt >= 1 && nxt < KT) {
                ok &= mbar_wait(smem_u32(done + (kt - 1) % ST), ((kt - 1) / ST) & 1);
                load(nxt, 3, true);
            }
        }
    }
    // every thread waits for the one-time barrier of the last commit, which
    // covers all MMAs (the stage barriers complete several phases each)
    ok &= mbar_wait(smem_u32(fin), 0);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

    // epilogue: the NS accumulators combine exactly in 64-bit integers, four
    // at a time (a0 2^21 + a1 2^14 + a2 2^7 + a3, |.| < 2^53), with one
    // conversion per four; the values go through shared memory (the pipeline
    // buffers are free now) so that the stores run along rows
    T *stage = reinterpret_cast<T *>(i8sm) + warp * 32 * (CW + 1);
    const double scale = ldexp(1.0, ea + eb - 33);
#pragma unroll 1
    for (int c8 = 0; c8 < CW / 8; c8++) {
        unsigned r[NS][8];
#pragma unroll
        for (int q = 0; q < NS; q++) {
            const unsigned taddr = tmem + ((unsigned)(32 * rq) << 16) + (unsigned)(q * BN + CW * ch + 8 * c8);
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                         : "=r"(r[q][0]), "=r"(r[q][1]), "=r"(r[q][2]), "=r"(r[q][3]),
                           "=r"(r[q][4]), "=r"(r[q][5]), "=r"(r[q][6]), "=r"(r[q][7])
                         : "r"(taddr));
        }
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int e = 0; e < 8; e++) {
            T v;
            const long long c = ((long long)(int)r[0][e] << 21) + ((long long)(int)r[1][e] << 14) +
                                ((long long)(int)r[2][e] << 7) + (long long)(int)r[3][e];
            if constexpr (NS == 4) {
                // x = c 2^(ea + eb - 33): exact up to the one rounding to FP32
                v = (T)((float)c * (float)scale);
            } else {
                const long long c2 = ((long long)(int)r[4][e] << 21) + ((long long)(int)r[5][e] << 14) +
                                     ((long long)(int)r[6][e] << 7) + (long long)(int)r[7][e];
                v = (T)(((double)c + ldexp((double)c2, -28)) * scale);
            }
            stage[lane * (CW + 1) + 8 * c8 + e] = ok ? v : (T)__int_as_float(0x7fc00000);
        }
    }
    __syncwarp();
    double part = 0;
    float vmax = 0.f;
#pragma unroll
    for (int it = 0; it < CW; it++) {
        const int e = it * 32 + lane, row = e / CW, col = e % CW;
        const int gm = m0 + 32 * rq + row, gn = n0 + CW * ch + col;
        if (gm >= M || gn >= N) continue;
        part += epi_apply<EPI, T>(go, grid_n, ge, gm, gn, stage[row * (CW + 1) + col],
                                  pre[it], vmax);
    }
    if (EPI != EPI_FIELD && batch.amax_out) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        if (lane == 0 && vmax > 0.f) atomicMax(batch.amax_out + g.prob, __float_as_uint(vmax));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                     :: "r"(tmem), "r"(Cfg::TMEM_COLS) : "memory");
    if (EPI == EPI_FIELD && go.kind == 3) bz_reduce<Cfg::THREADS>(part, go.bz_sum);
}

// ---------------------------------------------------------------------------
// Persistent, warp-specialised form of the transform waves.  One CTA per SM
// walks a static share of the wave's output tiles (every product of the wave
// in one list, tile t on CTA t mod grid).  Warp 0 streams the operand stages
// (one lane issues the bulk copies), warp 1 issues the MMAs, warps 4-11 read
// tensor memory, combine and store.
//
// Wide slice products: the B slices of a stage lie side by side in shared
// memory (slice j at columns j bn .. j bn + bn - 1 of one N-major operand), so
// the products of A slice i with B slices 0 .. NS-1-i are one MMA of
// N = (NS - i) bn columns whose accumulator starts at column block i: the
// product A_i B_j lands in block i + j, the accumulator of its weight.  NS
// MMAs of up to 256 columns (split where wider) replace NS (NS + 1) / 2
// narrow ones, and every A slice is read from shared memory once per MMA
// instead of once per B slice.
//
// Tensor memory holds 512 / (NS bn) accumulator sets: with four slices two
// sets alternate, so a tile's epilogue overlaps the next tile's main loop;
// with eight slices the one set is released as soon as the epilogue warps
// hold the combined values in registers, before they store them.
//
// The last tile column of a product narrower than a multiple of 64 uses a
// narrower tile (16, 32 or 48 columns): less operand traffic and fewer MMA
// columns for the padding.
// ---------------------------------------------------------------------------
constexpr int WP_BN = 64;                 // widest tile (columns)
constexpr int WP_EPI_WARP0 = 4;           // warps 4 .. 11 run the epilogue
constexpr int WP_EPI_WARPS = 8;
constexpr int WP_THREADS = 32 * (WP_EPI_WARP0 + WP_EPI_WARPS);

// KS k tiles (of 32) per pipeline stage: one barrier round trip and one
// commit per KS x NS wide MMAs.
template <int NS, int KS>
struct WPCfg {
    static constexpr int B_TILE = I8_BK * WP_BN;               // bytes per B slice (64 wide)
    static constexpr int KSTAGE = NS * (I8_A_SLICE + B_TILE);  // one k tile: 24 KB (4 slices) / 48 KB (8)
    static constexpr int STAGE = KS * KSTAGE;
    static constexpr int SET_COLS = NS * WP_BN;                // 256 / 512 TMEM columns
    static constexpr int NSETS = 512 / SET_COLS;               // 2 / 1 accumulator sets
    static constexpr int CW = WP_BN / 2;                       // epilogue columns per warp (max)
    // Per epilogue warp a 32 x CW block of outputs in shared memory (one
    // padding column), so that the stores run along rows.  (Storing straight
    // from registers, a lane per row, to make room for a fourth 48 KB FP64
    // stage measured 4 % slower at N = 513.)
    static constexpr bool STAGED = true;
    static constexpr int EPI_BYTES = STAGED ? WP_EPI_WARPS * 32 * (CW + 1) * NS : 0;
    static constexpr int ST = ((STAGED ? 144 : 192) * 1024) / STAGE;  // pipeline stages
    static_assert(ST >= 2, "at least two pipeline stages");
    static constexpr size_t smem = (size_t)ST * STAGE + EPI_BYTES + 256;
};

// Instruction descriptor of kind::i8 (s32 accumulator, signed int8 A K-major,
// B N-major), M = 128, N = n.
__device__ __forceinline__ unsigned i8_idesc_n(int n)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | (1u << 16) | ((unsigned)(n >> 3) << 17) |
           ((unsigned)(I8_BM >> 4) << 24);
}

// Tile t of the batch: product s, tile row mt, tile column nt (nt fastest,
// so that the tiles running together share their A row block in L2), from
// the products' first tiles `tstart` (shared memory).
template <typename T>
__device__ __forceinline__ void wave_tile(const GemmDesc<T> *sd, const int *tstart, int nsub, int t,
                                          int &s, int &mt, int &nt)
{
    s = 0;
    while (s + 1 < nsub && t >= tstart[s + 1]) s++;
    const int tn = ntiles(sd[s].N, WP_BN), r = t - tstart[s];
    mt = r / tn;
    nt = r - mt * tn;
}

// Width of tile column nt: 64, or the remaining columns rounded up to 16.
__device__ __forceinline__ int wave_tile_bn(int N, int nt)
{
    const int rem = N - nt * WP_BN;
    return rem >= WP_BN ? WP_BN : (rem + 15) & ~15;
}

// A bounded wait that also gives up as soon as another role of the CTA has
// given up (`bad` set), so that a failed protocol ends the kernel quickly.
__device__ __forceinline__ bool wp_wait(unsigned mbar, unsigned parity, volatile int *bad)
{
    for (int it = 0; it < (1 << 22); it++) {
        unsigned done;
        asm volatile("{\n.reg .pred P1;\nmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n"
                     "selp.b32 %0, 1, 0, P1;\n}\n"
                     : "=r"(done) : "r"(mbar), "r"(parity) : "memory");
        if (done) return true;
        if ((it & 255) == 255 && *bad) return false;
    }
    *bad = 1;
    return false;
}

__device__ __forceinline__ void mbar_arrive(unsigned mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(mbar) : "memory");
}

template <typename T, int EPI, int KS>
__global__ void __launch_bounds__(WP_THREADS, 1)
k_wave_i8p(const __grid_constant__ GemmBatch<T> batch, int total)
{
    constexpr int NS = Slices<T>::n;
    using Cfg = WPCfg<NS, KS>;
    constexpr int ST = Cfg::ST, NSETS = Cfg::NSETS, CW = Cfg::CW;
    extern __shared__ __align__(1024) uint8_t wpsm[];
    T *epi_stage = reinterpret_cast<T *>(wpsm + ST * Cfg::STAGE);          // epilogue blocks
    uint64_t *full = reinterpret_cast<uint64_t *>(wpsm + ST * Cfg::STAGE + Cfg::EPI_BYTES);  // [ST]
    uint64_t *empty = full + ST;                                            // [ST] stage consumed
    uint64_t *tfull = empty + ST;                                           // [NSETS] tile accumulated
    uint64_t *tempty = tfull + NSETS;                                       // [NSETS] set drained
    unsigned *tslot = reinterpret_cast<unsigned *>(tempty + NSETS);
    int *bad = reinterpret_cast<int *>(tslot + 1);                          // a bounded wait gave up

    // the products' descriptors and the field outputs, copied to shared
    // memory once: every role reads them per tile, and dynamically indexed
    // reads of the kernel parameters are slow and serialise
    __shared__ GemmDesc<T> sd[MAXSUB];
    __shared__ FieldOut so[NPROB];
    __shared__ int tstart[MAXSUB + 1];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    {
        const int *src = reinterpret_cast<const int *>(&batch.d[0]);
        int *dst = reinterpret_cast<int *>(sd);
        for (int i = tid; i < (int)(sizeof(sd) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
        const int *src2 = reinterpret_cast<const int *>(&batch.out[0]);
        int *dst2 = reinterpret_cast<int *>(so);
        for (int i = tid; i < (int)(sizeof(so) / sizeof(int)); i += blockDim.x) dst2[i] = src2[i];
        if (tid == 0) {
            int acc = 0;
            for (int q = 0; q < batch.nsub; q++) {
                tstart[q] = acc;
                acc += ntiles(batch.d[q].M, I8_BM) * ntiles(batch.d[q].N, WP_BN);
            }
            tstart[batch.nsub] = acc;
        }
    }
    const int nsub = batch.nsub, grid_n = batch.grid_n;
    unsigned *const amax_out = batch.amax_out;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tslot)), "r"(512) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int q = 0; q < 2 * ST + NSETS; q++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(full + q)), "r"(1)
                         : "memory");
        for (int q = 0; q < NSETS; q++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;"
                         :: "r"(smem_u32(tempty + q)), "r"(WP_EPI_WARPS) : "memory");
        *bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = *tslot;
    volatile int *vbad = bad;
    // every role reads or writes what the preceding kernels produce or read
    pdl_wait();
    pdl_trigger();

    if (warp == 0) {
        // ---- producer: two bulk copies per stage (A, B) ----
        unsigned g = 0;
        for (int t = blockIdx.x; t < total; t += gridDim.x) {
            int s, mt, nt;
            wave_tile(sd, tstart, nsub, t, s, mt, nt);
            const GemmDesc<T> &d = sd[s];
            const int KT = ntiles(d.K, TL_K), bn = wave_tile_bn(d.N, nt);
            // the NS slices of a tile, and the tiles along k, are contiguous:
            // one copy for A and one for B per stage (a narrow last tile
            // column copies its columns of each slice)
            const uint8_t *At = reinterpret_cast<const uint8_t *>(d.A) + (int64_t)mt * KT * NS * I8_A_SLICE;
            const uint8_t *Bt = reinterpret_cast<const uint8_t *>(d.B) + (int64_t)nt * KT * NS * Cfg::B_TILE;
            const unsigned bbytes = (unsigned)bn * I8_BK;
            for (int k0 = 0; k0 < KT; k0 += KS, g++) {
                const int ktn = KT - k0 < KS ? KT - k0 : KS;
                const int buf = (int)(g % ST);
                if (g >= (unsigned)ST) wp_wait(smem_u32(empty + buf), ((g / ST) - 1) & 1, vbad);
                if (lane == 0) {
                    const unsigned sA = smem_u32(wpsm + buf * Cfg::STAGE);
                    const unsigned sB = sA + KS * NS * I8_A_SLICE;
                    const unsigned mb = smem_u32(full + buf);
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;"
                                 :: "r"((unsigned)(ktn * NS) * (I8_A_SLICE + bbytes)), "r"(mb) : "memory");
                    bulk_g2s(sA, At + (int64_t)k0 * NS * I8_A_SLICE, ktn * NS * I8_A_SLICE, mb);
                    const uint8_t *Bk = Bt + (int64_t)k0 * NS * Cfg::B_TILE;
                    if (bn == WP_BN) {
                        bulk_g2s(sB, Bk, ktn * NS * Cfg::B_TILE, mb);
                    } else {
                        for (int q = 0; q < ktn * NS; q++)
                            bulk_g2s(sB + q * bbytes, Bk + q * Cfg::B_TILE, bbytes, mb);
                    }
                }
                __syncwarp();
            }
        }
        // the last fill of every buffer has landed before the CTA may exit
        for (int q = 0; q < ST && q < (int)g; q++) {
            const unsigned last = g - 1 - (unsigned)q;
            wp_wait(smem_u32(full + last % ST), (last / ST) & 1, vbad);
        }
    } else if (warp == 1) {
        // ---- MMA issue (lane 0; the warp follows the loop) ----
        unsigned g = 0;
        int lt = 0;
        for (int t = blockIdx.x; t < total; t += gridDim.x, lt++) {
            int s, mt, nt;
            wave_tile(sd, tstart, nsub, t, s, mt, nt);
            const GemmDesc<T> &d = sd[s];
            const int KT = ntiles(d.K, TL_K), bn = wave_tile_bn(d.N, nt);
            const int set = lt % NSETS;
            if (lt >= NSETS) wp_wait(smem_u32(tempty + set), ((lt / NSETS) - 1) & 1, vbad);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned acc = tmem + (unsigned)(set * Cfg::SET_COLS);
            const int per = 256 / bn;   // B slices per MMA at most
            const unsigned bstep = (unsigned)(NS * bn * I8_BK);   // one k tile of B slices
            for (int k0 = 0; k0 < KT; k0 += KS, g++) {
                const int ktn = KT - k0 < KS ? KT - k0 : KS;
                const int buf = (int)(g % ST);
                wp_wait(smem_u32(full + buf), (g / ST) & 1, vbad);
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                if (lane == 0) {
                    const unsigned a0 = smem_u32(wpsm + buf * Cfg::STAGE);
                    // descriptors of the stage's first A and B slices; a slice
                    // or k tile further is an addition to the start-address field
                    const uint64_t da0 = umma_desc(a0, 128, 256);
                    const uint64_t db0 = umma_desc(a0 + KS * NS * I8_A_SLICE, 128, 512);
                    for (int j = 0; j < ktn; j++) {
#pragma unroll
                    for (int i = 0; i < NS; i++) {
                        const uint64_t da = da0 + (uint64_t)((j * NS + i) * (I8_A_SLICE >> 4));
                        for (int j0 = 0; j0 < NS - i; j0 += per) {
                            const int nb = (NS - i - j0) < per ? (NS - i - j0) : per;
                            const uint64_t db = db0 + (uint64_t)((j * bstep + j0 * bn * I8_BK) >> 4);
                            const unsigned dcol = acc + (unsigned)((i + j0) * bn);
                            const unsigned en = (k0 > 0 || j > 0 || i > 0) ? 1u : 0u;
                            asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                                         "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, "
                                         "{%5, %5, %5, %5}, p;\n}\n"
                                         :: "r"(dcol), "l"(da), "l"(db), "r"(i8_idesc_n(nb * bn)),
                                            "r"(en), "r"(0u)
                                         : "memory");
                        }
                    }
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                                 :: "r"(smem_u32(empty + buf)) : "memory");
                    if (k0 + KS >= KT)
                        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                                     :: "r"(smem_u32(tfull + set)) : "memory");
                }
                __syncwarp();
            }
        }
    } else if (warp >= WP_EPI_WARP0) {
        // ---- epilogue: warp e reads TMEM lanes 32 (e % 4) .. (tile rows) and
        // the column half e / 4 of the tile into its shared-memory block (a
        // lane per row), then stores the block along rows (pass `it` of a
        // lane covers element it * 32 + lane of the 32 x cw block) ----
        const int e = warp - WP_EPI_WARP0, rq = e & 3, ch = e >> 2;
        T *blk = epi_stage + e * 32 * (CW + 1);
        int lt = 0;
        for (int t = blockIdx.x; t < total; t += gridDim.x, lt++) {
            int s, mt, nt;
            wave_tile(sd, tstart, nsub, t, s, mt, nt);
            // register copies of the tile's descriptor and field output: the
            // stores below could alias shared memory as far as the compiler
            // knows, so references into shared memory would be reloaded
            // after every store
            const GemmDesc<T> &ds = sd[s];
            EpiDesc<T> d;
            d.C = ds.C; d.E = ds.E; d.ldc = ds.ldc; d.lde = ds.lde; d.rmul = ds.rmul; d.radd = ds.radd;
            d.cmul = ds.cmul; d.cadd = ds.cadd; d.M = ds.M; d.N = ds.N;
            const int prob = ds.prob;
            const FieldOut o = so[prob];
            const int ea = operand_exp(ds.amax_a), eb = operand_exp(ds.amax_b);
            const int bn = wave_tile_bn(d.N, nt), cw = bn / 2;
            const int r0 = mt * I8_BM + 32 * rq, n0 = nt * WP_BN + ch * cw;
            const double scale = ldexp(1.0, ea + eb - 33);
            const int set = lt % NSETS;
            wp_wait(smem_u32(tfull + set), (lt / NSETS) & 1, vbad);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned acc = tmem + ((unsigned)(32 * rq) << 16) + (unsigned)(set * Cfg::SET_COLS);
            const bool poison = *vbad != 0;
            T vreg[Cfg::STAGED ? 1 : CW];
#pragma unroll
            for (int c8 = 0; c8 < CW / 8; c8++) {
                if (8 * c8 >= cw) break;
                unsigned r[NS][8];
#pragma unroll
                for (int q = 0; q < NS; q++) {
                    const unsigned taddr = acc + (unsigned)(q * bn + ch * cw + 8 * c8);
                    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                                 : "=r"(r[q][0]), "=r"(r[q][1]), "=r"(r[q][2]), "=r"(r[q][3]),
                                   "=r"(r[q][4]), "=r"(r[q][5]), "=r"(r[q][6]), "=r"(r[q][7])
                                 : "r"(taddr));
                }
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int x = 0; x < 8; x++) {
                    const long long c = ((long long)(int)r[0][x] << 21) + ((long long)(int)r[1][x] << 14) +
                                        ((long long)(int)r[2][x] << 7) + (long long)(int)r[3][x];
                    T v;
                    if constexpr (NS == 4) {
                        v = (T)((float)c * (float)scale);
                    } else {
                        const long long c2 = ((long long)(int)r[4][x] << 21) + ((long long)(int)r[5][x] << 14) +
                                             ((long long)(int)r[6][x] << 7) + (long long)(int)r[7][x];
                        v = (T)(((double)c + ldexp((double)c2, -28)) * scale);
                    }
                    if (poison) v = (T)__int_as_float(0x7fc00000);
                    if constexpr (Cfg::STAGED) blk[lane * (CW + 1) + 8 * c8 + x] = v;
                    else vreg[8 * c8 + x] = v;
                }
            }
            // the accumulators are in shared memory or registers: release the
            // set to the MMA warp
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(smem_u32(tempty + set));
            double part = 0;
            float vmax = 0.f;
            if constexpr (!Cfg::STAGED) {
                // a lane stores its row, eight columns at a time
                const int gm = r0 + lane;
#pragma unroll
                for (int c0 = 0; c0 < CW; c0 += 8) {
                    if (c0 >= cw) break;
                    double pre[8];
#pragma unroll
                    for (int x = 0; x < 8; x++)
                        pre[x] = (EPI != EPI_STORE && gm < d.M && n0 + c0 + x < d.N)
                                     ? epi_pre<EPI, T>(o, grid_n, d, gm, n0 + c0 + x) : 0.0;
#pragma unroll
                    for (int x = 0; x < 8; x++) {
                        if (gm >= d.M || n0 + c0 + x >= d.N) continue;
                        part += epi_apply<EPI, T>(o, grid_n, d, gm, n0 + c0 + x, vreg[c0 + x], pre[x], vmax);
                    }
                }
            }
            // stores along rows, eight passes at a time: the eight operands
            // the epilogue reads (spectral factors, previous fields) are
            // loaded together first
            for (int c0 = 0; Cfg::STAGED && c0 < cw; c0 += 8) {
                double pre[8];
#pragma unroll
                for (int x = 0; x < 8; x++) {
                    const int el = (c0 + x) * 32 + lane, row = el / cw, col = el - row * cw;
                    pre[x] = (EPI != EPI_STORE && r0 + row < d.M && n0 + col < d.N)
                                 ? epi_pre<EPI, T>(o, grid_n, d, r0 + row, n0 + col) : 0.0;
                }
#pragma unroll
                for (int x = 0; x < 8; x++) {
                    const int el = (c0 + x) * 32 + lane, row = el / cw, col = el - row * cw;
                    if (r0 + row >= d.M || n0 + col >= d.N) continue;
                    part += epi_apply<EPI, T>(o, grid_n, d, r0 + row, n0 + col, blk[row * (CW + 1) + col],
                                              pre[x], vmax);
                }
            }
            __syncwarp();   // the block is rewritten by the next tile
            if (EPI != EPI_FIELD && amax_out) {
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
                if (lane == 0 && vmax > 0.f) atomicMax(amax_out + prob, __float_as_uint(vmax));
            }
            if (EPI == EPI_FIELD && o.kind == 3) {
#pragma unroll
                for (int sh = 16; sh > 0; sh >>= 1) part += __shfl_xor_sync(0xffffffffu, part, sh);
                if (lane == 0) atomicAdd(o.bz_sum, part);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(512) : "memory");
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
    // mixed precision: the source's largest |element| (float bits); the
    // output is then written as packed int8 slices scaled by the bound 2x that
    const unsigned *src_max;
};

template <typename T>
struct FoldBatch {
    FoldDesc<T> d[NPROB];
    unsigned *clear;      // NPROB maxima zeroed here for the next producer, or NULL
};

// Slice fold: FP32 or FP64 source, tiled int8 slice planes out (zero
// padded, sizeof(T) planes).  Column folds feed right waves, so U (R x he)
// and V (R x ho) are stored in the A role; row folds feed left waves, so U
// (he x C) and V (ho x C) are stored in the B role.  A thread makes four
// consecutive elements along the contiguous direction of a core-matrix row
// (K for A, N for B): one 32-bit store per plane.
template <int NS, typename T>
__device__ __forceinline__ void put_slices4(uint8_t *blk, int64_t at, int stride, const T v[4],
                                            double scale)
{
    unsigned w[NS];
#pragma unroll
    for (int i = 0; i < NS; i++) w[i] = 0u;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        unsigned sl[NS];
        slices_biased(v[e], scale, sl);
#pragma unroll
        for (int i = 0; i < NS; i++) w[i] |= sl[i] << (8 * e);
    }
#pragma unroll
    for (int i = 0; i < NS; i++)
        *reinterpret_cast<unsigned *>(blk + at + (int64_t)i * stride) = __vsub4(w[i], 0x40404040u);
}

// One thread per 32-bit word of every slice plane (four consecutive
// elements): a warp covers a core matrix's eight rows (lanes 0-7) by four
// groups of four elements (lanes / 8), so that each of its stores writes
// 128 contiguous bytes per plane; the source elements are read straight from
// L2.  Column folds (A role, feeding right waves) pair element j with
// C - 1 - j of the same row; row folds (B role, feeding left waves) pair rows
// k and R - 1 - k.
constexpr int FOLD_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(FOLD_THREADS) k_fold_slices(const __grid_constant__ FoldBatch<T> fb)
{
    constexpr int NS = Slices<T>::n;
    pdl_wait();
    pdl_trigger();
    const FoldDesc<T> &f = fb.d[blockIdx.z];
    const int R = f.R, C = f.C, ldc = ld2(C);
    if (fb.clear && blockIdx.x == 0 && blockIdx.z == 0 && threadIdx.x < NPROB)
        fb.clear[threadIdx.x] = 0u;
    const int idx = blockIdx.x * FOLD_THREADS + threadIdx.x, lane = idx & 31, w = idx >> 5;
    uint8_t *blk = reinterpret_cast<uint8_t *>(f.dst);
    if (!f.by_rows) {
        const int he = (C + 1) / 2, ho = C - he, mid = (C - 1) / 2;
        const int KTu = ntiles(he, TL_K), KTv = ntiles(ho, TL_K);
        const int nu = 2 * KTu, nkb = nu + 2 * KTv;     // 16-wide k blocks of U, then of V
        const int rb = w / nkb, kb = w - rb * nkb;
        const int r = rb * 8 + (lane & 7);
        if (r >= ntiles(R, TL_M) * TL_M) return;
        const double scale = ldexp(1.0, -bound_exp(2.f * __uint_as_float(*f.src_max)));
        const bool isv = kb >= nu;
        const int k = (isv ? kb - nu : kb) * 16 + (lane >> 3) * 4;
        const T *x = f.src + (int64_t)(r < R ? r : 0) * ldc;
        T v[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int j = k + e;
            if (r >= R) v[e] = T(0);
            else if (!isv) v[e] = j < mid ? x[j] + x[C - 1 - j] : (j == mid ? x[mid] : T(0));
            else v[e] = j < ho ? x[j] - x[C - 1 - j] : T(0);
        }
        if (!isv) put_slices4<NS>(blk, a_tile_off(r, k, KTu, NS, 0), I8_A_SLICE, v, scale);
        else put_slices4<NS>(blk + NS * a_plane_bytes(R, he), a_tile_off(r, k, KTv, NS, 0), I8_A_SLICE,
                             v, scale);
    } else {
        const int he = (R + 1) / 2, ho = R - he, mid = (R - 1) / 2;
        const int KTu = ntiles(he, TL_K), KTv = ntiles(ho, TL_K);
        const int ng = ntiles(C, TL_N) * 4, ntask = 2 * ng;  // 16-wide n groups of U, then of V
        const int kb = w / ntask, t = w - kb * ntask;
        const int k = kb * 8 + (lane & 7);
        if (k >= KTu * TL_K) return;
        const bool isv = t >= ng;
        if (isv && k >= KTv * TL_K) return;
        const double scale = ldexp(1.0, -bound_exp(2.f * __uint_as_float(*f.src_max)));
        const int n = (isv ? t - ng : t) * 16 + (lane >> 3) * 4;
        const bool valid = isv ? k < ho : k < he;
        const T *ra = f.src + (int64_t)(valid ? k : 0) * ldc;
        const T *rb = f.src + (int64_t)(valid ? R - 1 - k : 0) * ldc;
        const bool single = !isv && k == mid;
        T v[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int c = n + e;
            v[e] = (!valid || c >= C) ? T(0) : (single ? ra[c] : (isv ? ra[c] - rb[c] : ra[c] + rb[c]));
        }
        if (!isv) put_slices4<NS>(blk, b_tile_off(k, n, KTu, NS, 0), TL_K * TL_N, v, scale);
        else put_slices4<NS>(blk + NS * b_plane_bytes(he, C), b_tile_off(k, n, KTv, NS, 0), TL_K * TL_N,
                             v, scale);
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
    double i2h, idxi, irb;                    // 1 / (2 h), 1 / dxi, 1 / rb_div
    const double *ro_f, *jx_f, *jy_f, *jz_f;  // full currents, n_f planes
    const double *ro_p, *jx_p, *jy_p, *jz_p;  // prev currents, n_p planes
    int n_f, n_p;
    const double *rb_full, *rb_prev;
    const double *Ex, *Ey, *Bx, *By;          // fields (Helmholtz term)
    double *bz_sum;
    unsigned *amax_out;                       // mixed: per-output max |value| (zeroed), or NULL
    int with_phi;
};

__device__ __forceinline__ double psum(const double *a, int np, int64_t plane, int64_t i)
{
    return np == 2 ? a[i] + a[i + plane] : a[i];
}

constexpr int RHS_TY = 8, RHS_TX = 32;

template <typename T>
__device__ __forceinline__ void rhs_node(const RhsArgs &a, const double (*s_ro)[RHS_TX + 2],
                                         const double (*s_jz)[RHS_TX + 2],
                                         const double (*s_jx)[RHS_TX + 2],
                                         const double (*s_jy)[RHS_TX + 2], int li, int lj, int i,
                                         int j, T *X0, T *X1, T *X2, T *X3, T *X4, T *X5, T *X6,
                                         float mx[NPROB])
{
    const int N = a.N, n = N - 2;
    const int ldN = ld2(N), ldn = ld2(n);
    const int64_t plane = (int64_t)N * N;
    const int64_t t = (int64_t)i * N + j;
    const bool inner = i >= 1 && i < N - 1 && j >= 1 && j < N - 1;
    double dro_dx = 0, dro_dy = 0, djz_dx = 0, djz_dy = 0;
    if (inner) {
        dro_dx = (s_ro[li + 1][lj] - s_ro[li - 1][lj]) * a.i2h;
        dro_dy = (s_ro[li][lj + 1] - s_ro[li][lj - 1]) * a.i2h;
        djz_dx = (s_jz[li + 1][lj] - s_jz[li - 1][lj]) * a.i2h;
        djz_dy = (s_jz[li][lj + 1] - s_jz[li][lj - 1]) * a.i2h;
    }
    const double djx_dxi = (psum(a.jx_p, a.n_p, plane, t) - s_jx[li][lj]) * a.idxi;
    const double djy_dxi = (psum(a.jy_p, a.n_p, plane, t) - s_jy[li][lj]) * a.idxi;
    const double Ex_rhs = -(dro_dx - djx_dxi - a.c * a.Ex[t]);
    const double Ey_rhs = -(dro_dy - djy_dxi - a.c * a.Ey[t]);
    const double Bx_rhs = +(djz_dy - djy_dxi + a.c * a.Bx[t]);
    const double By_rhs = -(djz_dx - djx_dxi - a.c * a.By[t]);
    if (i >= 1 && i < N - 1) {
        const int64_t o = (int64_t)(i - 1) * ldN + j;
        X0[o] = (T)Ey_rhs; mx[0] = fmaxf(mx[0], abs_bound((T)Ey_rhs));
        X1[o] = (T)Bx_rhs; mx[1] = fmaxf(mx[1], abs_bound((T)Bx_rhs));
    }
    if (j >= 1 && j < N - 1) {
        const int64_t o = (int64_t)i * ldn + (j - 1);
        X2[o] = (T)Ex_rhs; mx[2] = fmaxf(mx[2], abs_bound((T)Ex_rhs));
        X3[o] = (T)By_rhs; mx[3] = fmaxf(mx[3], abs_bound((T)By_rhs));
    }
    double djx_dy = 0, djy_dx = 0;
    if (inner) {
        djx_dy = s_jx[li][lj + 1] - s_jx[li][lj - 1];
        djy_dx = s_jy[li + 1][lj] - s_jy[li - 1][lj];
    }
    const double bz_rhs = -(djx_dy - djy_dx) * a.i2h;
    X6[(int64_t)i * ldN + j] = (T)bz_rhs;
    mx[6] = fmaxf(mx[6], abs_bound((T)bz_rhs));
    if (inner) {
        const int64_t o = (int64_t)(i - 1) * ldn + (j - 1);
        const double djx_dx = s_jx[li + 1][lj] - s_jx[li - 1][lj];
        const double djy_dy = s_jy[li][lj + 1] - s_jy[li][lj - 1];
        const double ez_rhs = -(djx_dx + djy_dy) * a.i2h;
        X4[o] = (T)ez_rhs;
        mx[4] = fmaxf(mx[4], abs_bound((T)ez_rhs));
        if (a.with_phi) {
            const double phi_rhs = psum(a.ro_f, a.n_f, plane, t) - psum(a.jz_f, a.n_f, plane, t);
            X5[o] = (T)phi_rhs;
            mx[5] = fmaxf(mx[5], abs_bound((T)phi_rhs));
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(RHS_TX * RHS_TY)
k_fields_rhs(RhsArgs a, T *X0, T *X1, T *X2, T *X3, T *X4, T *X5, T *X6)
{
    pdl_wait();
    pdl_trigger();
    __shared__ double s_ro[RHS_TY + 2][RHS_TX + 2], s_jz[RHS_TY + 2][RHS_TX + 2];
    __shared__ double s_jx[RHS_TY + 2][RHS_TX + 2], s_jy[RHS_TY + 2][RHS_TX + 2];
    const int N = a.N;
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
            const double rbf = a.rb_full[q] * a.irb, rbp = a.rb_prev[q] * a.irb;
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
    float mx[NPROB] = {0, 0, 0, 0, 0, 0, 0};
    if (i < N && j < N) rhs_node(a, s_ro, s_jz, s_jx, s_jy, li, lj, i, j, X0, X1, X2, X3, X4, X5, X6, mx);
    if (a.amax_out) {
        // per-block maxima first: one atomic per block and problem
        __shared__ float s_mx[RHS_TY][NPROB];
#pragma unroll
        for (int p = 0; p < NPROB; p++) {
            float v = mx[p];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
            if (threadIdx.x == 0) s_mx[threadIdx.y][p] = v;
        }
        __syncthreads();
        if (threadIdx.y == 0 && threadIdx.x < NPROB) {
            float v = 0.f;
#pragma unroll
            for (int y = 0; y < RHS_TY; y++) v = fmaxf(v, s_mx[y][threadIdx.x]);
            if (v > 0.f) atomicMax(a.amax_out + threadIdx.x, __float_as_uint(v));
        }
    }
}

// Zero the per-problem operand maxima (a kernel rather than a memset, so that
// the chain of programmatic launches stays unbroken).
__global__ void k_clear_maxima(unsigned *m)
{
    pdl_wait();
    pdl_trigger();
    if (threadIdx.x < NPROB) m[threadIdx.x] = 0u;
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
    pdl_wait();
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
    unsigned *amax[2];    // per-problem operand maxima, alternating between folds
};

// A workspace slot holds one problem's matrix: natural rows of up to N + 4
// elements, or the tiled int8 slice planes of a folded matrix.
template <typename T>
static size_t slot_elems(int N)
{
    // the sizeof(T) tiled slice planes of both fold halves take at most
    // (N + 127) x (N + 64) bytes each, i.e. that many elements of T
    const size_t e = (size_t)(N + 128) * (N + 64);
    return (e + 31) / 32 * 32;
}

template <typename T>
static size_t work_bytes(int N)
{
    size_t b = 2 * NPROB * slot_elems<T>(N) * sizeof(T);
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
    for (int i = 0; i < NPROB; i++) { w.S1[i] = p; p += slot_elems<T>(N); }
    for (int i = 0; i < NPROB; i++) { w.S2[i] = p; p += slot_elems<T>(N); }
    size_t off = 2 * NPROB * slot_elems<T>(N) * sizeof(T);
    off = (off + 255) / 256 * 256;
    char *base = static_cast<char *>(ws);
    w.bz_raw = reinterpret_cast<double *>(base + off);
    off += (size_t)N * N * sizeof(double);
    off = (off + 255) / 256 * 256;
    w.bz_sum = reinterpret_cast<double *>(base + off);
    // the last 256 bytes: bz_sum, then two arrays of NPROB maxima
    w.amax[0] = reinterpret_cast<unsigned *>(base + off + 64);
    w.amax[1] = reinterpret_cast<unsigned *>(base + off + 128);
    return w;
}

template <typename T, int EPI>
static int launch_i8(const GemmBatch<T> &b, int nsub, int maxM, int maxN, cudaStream_t st)
{
    // 256 tensor-memory columns per CTA (NS accumulators x BN), two CTAs per
    // SM: 64-wide tiles for four slices, 32-wide for eight (128-wide tiles,
    // one CTA per SM, read less operand data but ran no faster)
    constexpr int BN = Slices<T>::n == 8 ? 32 : 64;
    using Cfg = I8Cfg<Slices<T>::n, BN>;
    static std::atomic<unsigned long long> attr{0};
    {
        const cudaError_t e = ensure_smem(k_gemm_i8<T, BN, EPI>, Cfg::smem, attr);
        if (e != cudaSuccess) return cuda_check(e, "i8 gemm smem attribute");
    }
    dim3 grid((maxN + BN - 1) / BN, (maxM + I8_BM - 1) / I8_BM, nsub);
    const cudaError_t e = launch_after(k_gemm_i8<T, BN, EPI>, grid, dim3(Cfg::THREADS), Cfg::smem, st, b);
    if (e != cudaSuccess) return cuda_check(e, "i8 gemm launch");
    return LCB_OK;
}

template <typename T, int EPI, int KS>
static int launch_wave_ks(GemmBatch<T> b, int nsub, cudaStream_t st)
{
    using Cfg = WPCfg<Slices<T>::n, KS>;
    static std::atomic<unsigned long long> attr{0};
    {
        const cudaError_t e = ensure_smem(k_wave_i8p<T, EPI, KS>, Cfg::smem, attr);
        if (e != cudaSuccess) return cuda_check(e, "persistent wave smem attribute");
    }
    b.nsub = nsub;
    int total = 0;
    for (int s = 0; s < nsub; s++) total += ntiles(b.d[s].M, I8_BM) * ntiles(b.d[s].N, WP_BN);
    if (total == 0) return LCB_OK;
    const int grid = total < sm_count() ? total : sm_count();
    const cudaError_t e = launch_after(k_wave_i8p<T, EPI, KS>, dim3(grid), dim3(WP_THREADS), Cfg::smem,
                                       st, b, total);
    if (e != cudaSuccess) return cuda_check(e, "persistent wave launch");
    return LCB_OK;
}

// k tiles per pipeline stage: LCB_WAVE_KS (1 or 2) if set, else 1 in FP64
// (a 48 KB stage) and 2 in mixed precision (two 24 KB k tiles).
static int wave_ks(int ns)
{
    static const int env = [] {
        const char *v = getenv("LCB_WAVE_KS");
        return v ? atoi(v) : 0;
    }();
    if (env == 1 || env == 2) return env;
    return ns == 8 ? 1 : 2;
}

template <typename T, int EPI>
static int launch_wave_p(const GemmBatch<T> &b, int nsub, cudaStream_t st)
{
    if constexpr (Slices<T>::n == 4)
        if (wave_ks(4) == 2) return launch_wave_ks<T, EPI, 2>(b, nsub, st);
    return launch_wave_ks<T, EPI, 1>(b, nsub, st);
}

// The two forms of the transform waves: one CTA per output tile, or the
// persistent warp-specialised kernel.  Which one runs for a grid and
// precision is measured (wave_kernel_for below).
enum { WK_TILED = 1, WK_PERSISTENT = 2 };

template <typename T>
static int launch_wave(const GemmBatch<T> &b, int nsub, int epi, int maxM, int maxN,
                       int wk, cudaStream_t st)
{
    if (wk == WK_PERSISTENT) {
        if (epi == EPI_STORE) return launch_wave_p<T, EPI_STORE>(b, nsub, st);
        if (epi == EPI_SCALE) return launch_wave_p<T, EPI_SCALE>(b, nsub, st);
        return launch_wave_p<T, EPI_FIELD>(b, nsub, st);
    }
    if (epi == EPI_STORE) return launch_i8<T, EPI_STORE>(b, nsub, maxM, maxN, st);
    if (epi == EPI_SCALE) return launch_i8<T, EPI_SCALE>(b, nsub, maxM, maxN, st);
    return launch_i8<T, EPI_FIELD>(b, nsub, maxM, maxN, st);
}

template <typename T>
static int run_wave(const GemmBatch<T> &b, int nsub, int epi, int wk, cudaStream_t st,
                    const char *what)
{
    int maxM = 0, maxN = 0;
    for (int s = 0; s < nsub; s++) {
        maxM = b.d[s].M > maxM ? b.d[s].M : maxM;
        maxN = b.d[s].N > maxN ? b.d[s].N : maxN;
    }
    const int rc = launch_wave(b, nsub, epi, maxM, maxN, wk, st);
    if (rc) return rc;
    LCB_LAUNCH_CHECK(what);
    return LCB_OK;
}

template <typename T>
static int run_fold(T *const *src, T *const *dst, const int *probs, int np, const int *rows,
                    const int *cols, int by_rows, int N, cudaStream_t st,
                    const unsigned *src_max, unsigned *clear)
{
    LCB_REQUIRE(src_max, "fold without operand maxima");
    FoldBatch<T> fb;
    memset(&fb, 0, sizeof(fb));
    for (int q = 0; q < np; q++) {
        const int p = probs[q];
        fb.d[q].src = src[p];
        fb.d[q].dst = dst[p];
        fb.d[q].R = rows[p];
        fb.d[q].C = cols[p];
        fb.d[q].by_rows = by_rows;
        fb.d[q].src_max = src_max ? src_max + p : nullptr;
    }
    fb.clear = clear;
    // threads per problem: one per slice word of the largest problem (rows
    // padded to 8, words of 4 elements)
    const int he = (N + 1) / 2;
    const int64_t words = by_rows
        ? (int64_t)ntiles(he, TL_K) * TL_K * ntiles(N, TL_N) * TL_N * 2 / 4
        : (int64_t)ntiles(N, TL_M) * TL_M * ntiles(he, TL_K) * TL_K * 2 / 4;
    dim3 grid((unsigned)((words + FOLD_THREADS - 1) / FOLD_THREADS), 1u, np);
    const cudaError_t e = launch_after(k_fold_slices<T>, grid, dim3(FOLD_THREADS), 0, st, fb);
    if (e != cudaSuccess) return cuda_check(e, "fold launch");
    LCB_LAUNCH_CHECK("k_fold_slices");
    return LCB_OK;
}

template <typename T>
static int solve(const lcb_compute_fields_args *a, const T *ops, cudaStream_t st, int wk)
{
    const int N = a->grid_steps, n = N - 2;
    const OpLayout L = op_layout(N);
    Work<T> w = carve<T>(a->workspace, N);
    // Phi (problem 5) is skipped when neither of its outputs is wanted.
    const bool with_phi = a->out_half.f[6] || a->out_full.f[6];

    RhsArgs r;
    r.N = N; r.h = a->h; r.dxi = a->xi_step; r.c = a->subtraction_coeff;
    r.rb_div = a->rho_beam_divisor;
    // the kernel multiplies by reciprocals (at most an ulp from the quotients)
    r.i2h = 1.0 / (2.0 * a->h); r.idxi = 1.0 / a->xi_step; r.irb = 1.0 / a->rho_beam_divisor;
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
    // mixed precision: every producer of a matrix that a fold turns into
    // int8 slices (the right-hand sides, waves 1-3) records its largest
    // element per problem; the maxima alternate between two arrays, each
    // fold clearing the one that the next wave fills
    constexpr bool rec = true;
    unsigned *const mx0 = rec ? w.amax[0] : nullptr, *const mx1 = rec ? w.amax[1] : nullptr;
    unsigned *cur_mx = nullptr;
    r.amax_out = mx0;
    if (rec) {
        cudaError_t e = launch_after(k_clear_maxima, dim3(1), dim3(32), 0, st, mx0);
        if (e != cudaSuccess) return cuda_check(e, "clear maxima");
        count_launch();
    }
    {
        dim3 grid((N + RHS_TX - 1) / RHS_TX, (N + RHS_TY - 1) / RHS_TY);
        cudaError_t e = launch_after(k_fields_rhs<T>, grid, dim3(RHS_TX, RHS_TY), 0, st, r,
                                     w.S1[0], w.S1[1], w.S1[2], w.S1[3], w.S1[4], w.S1[5], w.S1[6]);
        if (e != cudaSuccess) return cuda_check(e, "rhs launch");
        count_launch();
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
                d.const_op = 2;
                d.M = rows[p]; d.K = par ? ho : he; d.N = par ? ho : he;
                d.rmul = 1; d.radd = 0; d.cmul = 2; d.cadd = par;
                d.C = w.S1[p]; d.ldc = ld2(C); d.prob = p;
                d.amax_a = cur_mx ? cur_mx + p : nullptr;
                if (rec) {
                    // tiled slice planes (A role): U block, then V block
                    const uint8_t *base = reinterpret_cast<const uint8_t *>(w.S2[p]);
                    d.A = reinterpret_cast<const T *>(base + (par ? Slices<T>::n * a_plane_bytes(rows[p], he) : 0));
                }
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
                d.const_op = 1;
                d.B = w.S2[p] + (par ? (int64_t)he * ld2(cols[p]) : 0); d.ldb = ld2(cols[p]);
                d.M = par ? ho : he; d.K = par ? ho : he; d.N = cols[p];
                d.rmul = 2; d.radd = par; d.cmul = 1; d.cadd = 0;
                if (!to_fields) { d.C = w.S1[p]; d.ldc = ld2(cols[p]); }
                d.E = op(mat[p]); d.lde = (int)L.ld[mat[p]];
                d.prob = p;
                d.amax_b = cur_mx ? cur_mx + p : nullptr;
                if (rec) {
                    // tiled slice planes (B role): U block, then V block
                    const uint8_t *base = reinterpret_cast<const uint8_t *>(w.S2[p]);
                    d.B = reinterpret_cast<const T *>(base + (par ? Slices<T>::n * b_plane_bytes(he, cols[p]) : 0));
                }
            }
        }
        return s;
    };

    int rc;
    // wave 1: S1 = S1 R
    if ((rc = run_fold<T>(w.S1, w.S2, probs, np, rows, cols, 0, N, st, mx0, mx1))) return rc;
    cur_mx = mx0;
    b.amax_out = mx1;
    if ((rc = run_wave<T>(b, right_wave(), EPI_STORE, wk, st, "wave1"))) return rc;
    // wave 2: S1 = (L S1) o Mat
    if ((rc = run_fold<T>(w.S1, w.S2, probs, np, rows, cols, 1, N, st, mx1, mx0))) return rc;
    cur_mx = mx1;
    b.amax_out = mx0;
    if ((rc = run_wave<T>(b, left_wave(false), EPI_SCALE, wk, st, "wave2"))) return rc;
    // wave 3: S1 = S1 R
    if ((rc = run_fold<T>(w.S1, w.S2, probs, np, rows, cols, 0, N, st, mx0, mx1))) return rc;
    cur_mx = mx0;
    b.amax_out = mx1;
    if ((rc = run_wave<T>(b, right_wave(), EPI_STORE, wk, st, "wave3"))) return rc;
    // wave 4: fields = L S1
    if ((rc = run_fold<T>(w.S1, w.S2, probs, np, rows, cols, 1, N, st, mx1, mx0))) return rc;
    cur_mx = mx1;
    b.amax_out = nullptr;
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
    if ((rc = run_wave<T>(b, nsub, EPI_FIELD, wk, st, "wave4"))) return rc;

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
        const cudaError_t e = launch_after(k_fields_finish, dim3(blocks), dim3(256), 0, st, fa);
        if (e != cudaSuccess) return cuda_check(e, "fields finish launch");
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
    const int sblocks = (int)((L.off[OP_D] + 255) / 256);
    // spectral matrices in the solver's precision, then the transform blocks
    // as int8 slice planes (four for FP32 operands, eight for FP64)
    if (precision == LCB_PREC_MIXED) {
        k_build_ops<float><<<blocks, 256, 0, as_stream(stream)>>>(
            N, h, subtraction_coeff, L, static_cast<float *>(operators));
        LCB_LAUNCH_CHECK("k_build_ops");
        k_build_slices<4><<<sblocks, 256, 0, as_stream(stream)>>>(N, L, static_cast<uint8_t *>(operators));
    } else {
        k_build_ops<double><<<blocks, 256, 0, as_stream(stream)>>>(
            N, h, subtraction_coeff, L, static_cast<double *>(operators));
        LCB_LAUNCH_CHECK("k_build_ops");
        k_build_slices<8><<<sblocks, 256, 0, as_stream(stream)>>>(N, L, static_cast<uint8_t *>(operators));
    }
    LCB_LAUNCH_CHECK("k_build_slices");
    return LCB_OK;
}

extern "C" size_t lcb_compute_fields_workspace_bytes(int grid_steps, int precision)
{
    if (grid_steps < 5) return 0;
    return precision == LCB_PREC_MIXED ? work_bytes<float>(grid_steps)
                                       : work_bytes<double>(grid_steps);
}

// ---------------------------------------------------------------------------
// Wave-kernel autotuner.  The first compute_fields of a (device, grid,
// precision) that is not being captured into a graph times the solve with
// each wave kernel (two warm-up and three timed calls each, CUDA events on
// the caller's stream) and keeps the faster; calls under capture before that
// use the one that measured faster on B200 at N = 513 (persistent for FP64,
// one tile per CTA for mixed precision).  The tuning calls compute the same
// outputs as the call itself (compute_fields only reads its inputs), so the
// call's result is unchanged.  LCB_WAVE_KERNEL=tiled or =persistent fixes the
// choice for every grid.
// ---------------------------------------------------------------------------
#include <map>
#include <mutex>
#include <tuple>

namespace lcb {

static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int>, int> g_tuned;   // (device, N, precision) -> WK_*

static int wave_kernel_env()
{
    static const int mode = [] {
        const char *v = getenv("LCB_WAVE_KERNEL");
        if (v && strcmp(v, "tiled") == 0) return (int)WK_TILED;
        if (v && strcmp(v, "persistent") == 0) return (int)WK_PERSISTENT;
        return 0;
    }();
    return mode;
}

template <typename T>
static int solve_tuned(const lcb_compute_fields_args *a, const T *ops, cudaStream_t st)
{
    const int fixed = wave_kernel_env();
    if (fixed) return solve<T>(a, ops, st, fixed);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_check(e, "cudaGetDevice");
    const auto key = std::make_tuple(dev, a->grid_steps, a->precision);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) return solve<T>(a, ops, st, it->second);
    }
    const int fallback = Slices<T>::n == 8 ? WK_PERSISTENT : WK_TILED;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return cuda_check(e, "cudaStreamIsCapturing");
    if (cs != cudaStreamCaptureStatusNone) return solve<T>(a, ops, st, fallback);
    cudaEvent_t ev[2];
    if ((e = cudaEventCreate(&ev[0])) != cudaSuccess) return cuda_check(e, "tuner event");
    if ((e = cudaEventCreate(&ev[1])) != cudaSuccess) {
        cudaEventDestroy(ev[0]);
        return cuda_check(e, "tuner event");
    }
    const int cand[2] = {WK_TILED, WK_PERSISTENT};
    float best = 0.f;
    int pick = fallback, rc = LCB_OK;
    for (int c = 0; c < 2 && rc == LCB_OK; c++) {
        for (int r = 0; r < 2 && rc == LCB_OK; r++) rc = solve<T>(a, ops, st, cand[c]);
        if (rc) break;
        cudaEventRecord(ev[0], st);
        for (int r = 0; r < 3 && rc == LCB_OK; r++) rc = solve<T>(a, ops, st, cand[c]);
        cudaEventRecord(ev[1], st);
        if (rc) break;
        if ((e = cudaEventSynchronize(ev[1])) != cudaSuccess) { rc = cuda_check(e, "tuner sync"); break; }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev[0], ev[1]);
        if (c == 0 || ms < best) { best = ms; pick = cand[c]; }
    }
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
    if (rc) return rc;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tuned[key] = pick;
    }
    return solve<T>(a, ops, st, pick);
}

}  // namespace lcb

extern "C" int lcb_wave_kernel_choice(int grid_steps, int precision)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    std::lock_guard<std::mutex> lock(lcb::g_tune_mu);
    auto it = lcb::g_tuned.find(std::make_tuple(dev, grid_steps, precision));
    return it == lcb::g_tuned.end() ? 0 : it->second;
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
        return solve_tuned<float>(a, static_cast<const float *>(a->operators), st);
    LCB_REQUIRE(a->precision == LCB_PREC_FP64, "bad precision %d", a->precision);
    return solve_tuned<double>(a, static_cast<const double *>(a->operators), st);
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
                "allocation-free entry point has %zu (largest grid: 283 in FP64, "
                "427 in mixed precision) -- use lcb_compute_fields with a workspace",
                a->grid_steps, a->precision, need, (size_t)LCB_NOALLOC_FIELDS_SCRATCH_BYTES);
    void *scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;
    lcb_compute_fields_args b = *a;
    b.workspace = scratch;
    b.workspace_bytes = LCB_NOALLOC_FIELDS_SCRATCH_BYTES;
    return lcb_compute_fields(&b, stream);
}
