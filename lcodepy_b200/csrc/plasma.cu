// Plasma particle kernels: free-streaming estimate, fused gather + push, and
// tiled charge/current deposition.  FP64 particles (SoA, coalesced).
#include <type_traits>

#include "common.cuh"

namespace lcb {

// ---------------------------------------------------------------------------
// K1: copy prev -> full and free-stream (lcode/plasma3d/move.py:292-313,
// copy at :337-339).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_move_wo_fields(int64_t n, double xi_step, const double *__restrict__ m,
                 const double *__restrict__ xo_p, const double *__restrict__ yo_p,
                 const double *__restrict__ px_p, const double *__restrict__ py_p,
                 const double *__restrict__ pz_p, const double *__restrict__ q_p,
                 double *xo_f, double *yo_f, double *px_f, double *py_f,
                 double *pz_f, double *q_f)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const double mk = m[k], px = px_p[k], py = py_p[k], pz = pz_p[k];
        double xo = xo_p[k], yo = yo_p[k];
        if (mk != 0) {
            const double gm = sqrt(mk * mk + pz * pz + px * px + py * py);
            const double adv = xi_step / (gm - pz);
            xo += px * adv;
            yo += py * adv;
        }
        xo_f[k] = xo; yo_f[k] = yo;
        px_f[k] = px; py_f[k] = py; pz_f[k] = pz;
        q_f[k] = q_p[k];
    }
}

// ---------------------------------------------------------------------------
// K2: fused midpoint gather + two-pass momentum update + advance +
// reflection + absorption (lcode/plasma3d/move.py:169-289).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void reflect(double &x, double b, double &px, double &py, double &pz)
{
    if (x > b)  { x =  2 * b - x; px = py = pz = 0; }
    if (x < -b) { x = -2 * b - x; px = py = pz = 0; }
}

__global__ void __launch_bounds__(256)
k_move_smart(int64_t n, double xi_step, double boundary, double h, int N,
             const double *__restrict__ Exf, const double *__restrict__ Eyf,
             const double *__restrict__ Ezf, const double *__restrict__ Bxf,
             const double *__restrict__ Byf, const double *__restrict__ Bzf,
             const double *__restrict__ x_init, const double *__restrict__ y_init,
             const double *__restrict__ xo_p, const double *__restrict__ yo_p,
             const double *__restrict__ px_p, const double *__restrict__ py_p,
             const double *__restrict__ pz_p, const double *__restrict__ m,
             double *q_f, double *xo_f, double *yo_f, double *px_f,
             double *py_f, double *pz_f, int *err)
{
    const int half_n = N / 2;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const double qk = q_f[k];
        if (qk == 0) continue;
        const double xi0 = x_init[k], yi0 = y_init[k];
        const double opx = px_p[k], opy = py_p[k], opz = pz_p[k];
        double px = opx, py = opy, pz = opz;
        double xh = xi0 + (xo_p[k] + xo_f[k]) / 2;
        double yh = yi0 + (yo_p[k] + yo_f[k]) / 2;
        // The reference zeroes momenta when the midpoint is reflected; the
        // zeroed values only feed gamma in the first pass below.
        if (xh > boundary)  { xh =  2 * boundary - xh; px = py = pz = 0; }
        if (xh < -boundary) { xh = -2 * boundary - xh; px = py = pz = 0; }
        if (yh > boundary)  { yh =  2 * boundary - yh; px = py = pz = 0; }
        if (yh < -boundary) { yh = -2 * boundary - yh; px = py = pz = 0; }

        double xl, yl;
        const int ix = cell_of(xh / h + 0.5, half_n, xl);
        const int iy = cell_of(yh / h + 0.5, half_n, yl);
        double Ex = 0, Ey = 0, Ez = 0, Bx = 0, By = 0, Bz = 0;
        if (ix >= 2 && ix < N - 2 && iy >= 2 && iy < N - 2) {
            double wx[5], wy[5];
            weights4(xl, wx);
            weights4(yl, wy);
#pragma unroll
            for (int a = 0; a < 5; a++) {
                const int row = (ix + a - 2) * N + iy - 2;
#pragma unroll
                for (int b = 0; b < 5; b++) {
                    const double w = wx[a] * wy[b];
                    const int idx = row + b;
                    Ex += __ldg(Exf + idx) * w; Bx += __ldg(Bxf + idx) * w;
                    Ey += __ldg(Eyf + idx) * w; By += __ldg(Byf + idx) * w;
                    Ez += __ldg(Ezf + idx) * w; Bz += __ldg(Bzf + idx) * w;
                }
            }
        } else if (err) {
            atomicOr(err, LCB_DEVERR_PLASMA_STENCIL);
        }
        const double mk = m[k];
        // velocities as p * (1/gamma m): one quotient per pass instead of three
        double gm = sqrt(mk * mk + px * px + py * py + pz * pz);
        double ig = 1.0 / gm;
        double vx = px * ig, vy = py * ig, vz = pz * ig;
        double f = qk * xi_step / (1 - vz);
        double dpx = f * (Ex + vy * Bz - vz * By);
        double dpy = f * (Ey - vx * Bz + vz * Bx);
        double dpz = f * (Ez + vx * By - vy * Bx);
        px = opx + dpx * 0.5; py = opy + dpy * 0.5; pz = opz + dpz * 0.5;

        gm = sqrt(mk * mk + px * px + py * py + pz * pz);
        ig = 1.0 / gm;
        vx = px * ig; vy = py * ig; vz = pz * ig;
        f = qk * xi_step / (1 - vz);
        dpx = f * (Ex + vy * Bz - vz * By);
        dpy = f * (Ey - vx * Bz + vz * Bx);
        dpz = f * (Ez + vx * By - vy * Bx);
        px = opx + dpx * 0.5; py = opy + dpy * 0.5; pz = opz + dpz * 0.5;

        gm = sqrt(mk * mk + px * px + py * py + pz * pz);
        const double adv = xi_step / (gm - pz);
        double xo = xo_p[k] + px * adv;
        double yo = yo_p[k] + py * adv;
        px = opx + dpx; py = opy + dpy; pz = opz + dpz;

        double x = xi0 + xo, y = yi0 + yo;
        if (x > boundary)  { x =  2 * boundary - x; xo = x - xi0; px = py = pz = 0; }
        if (x < -boundary) { x = -2 * boundary - x; xo = x - xi0; px = py = pz = 0; }
        if (y > boundary)  { y =  2 * boundary - y; yo = y - yi0; px = py = pz = 0; }
        if (y < -boundary) { y = -2 * boundary - y; yo = y - yi0; px = py = pz = 0; }
        if (x >= boundary || x <= -boundary || y >= boundary || y <= -boundary) {
            xo = yo = 0; px = py = pz = 0;
            q_f[k] = 0;
        }
        xo_f[k] = xo; yo_f[k] = yo;
        px_f[k] = px; py_f[k] = py; pz_f[k] = pz;
    }
}

// ---------------------------------------------------------------------------
// K3: deposition (lcode/plasma3d/weights.py:151-190, 249-285).
//
// A block owns a TI x TJ tile of one sort's particle lattice (particles are
// created on a lattice, k = s*Np + i*Ns + j, and drift little per xi step, so
// a tile's particles stay in a compact cell window).  Contributions whose
// whole 5x5 stencil lies inside the block's shared-memory window [wx0, wx0+WX)
// x [wy0, wy0+WY) are accumulated there with shared atomics; any other
// particle (a runaway, a lattice that is not a lattice) goes straight to
// global atomics.  The window is then flushed with one global atomic per
// non-zero cell and quantity.  The window origin follows the tile's first
// particle's initial position, with S cells of slack for drift.
//
// FP64 shared atomics retry when two lanes of a warp hit the same address in
// the same instruction.  With two particles per cell along each axis (the
// 2 x 2 per cell lattice) the lanes of a warp are therefore given particles of
// one parity sub-lattice (every other row and column), which sit in distinct
// cells; all 25 stencil points of a warp instruction then differ too.
// ---------------------------------------------------------------------------
constexpr int DEP_TI = 16, DEP_TJ = 32, DEP_THREADS = 256;
constexpr int DEP_NP = DEP_TI * DEP_TJ;
constexpr int DEP_PPT = DEP_NP / DEP_THREADS;
constexpr int DEP_SLACK = 4;
constexpr int DEP_WX = 28, DEP_WY = 44;  // >= tile cells (fineness 1) + 4 + 2*slack

// Tile position (ti, tj) of the q-th particle slot of a block.
__device__ __forceinline__ void tile_slot(int q, bool two_per_cell, int &ti, int &tj)
{
    if (two_per_cell) {
        const int par = q >> 7, w = q & 127;        // 4 parity sub-lattices of 8 x 16
        ti = 2 * (w >> 4) + (par >> 1);
        tj = 2 * (w & 15) + (par & 1);
    } else {
        ti = q / DEP_TJ;
        tj = q % DEP_TJ;
    }
}

// Deposit one particle's 25-point stencil (weights.py:151-190 arithmetic)
// into the block's shared window, or straight into HBM when the stencil
// leaves the window.  dep = false: nothing to deposit.
// Accumulator of the mixed-precision deposit: every contribution is rounded
// to a multiple of 2^-32 and summed as a 64-bit integer, so the sums are
// exact and do not depend on the order of the atomics (an FP32 sum of the
// ~100 contributions a cell receives rounds at the magnitude of the running
// total, which for the electron density is the background ~1, and leaves a
// systematic ~1e-7 error that the background ions then expose).
//
// The rounding is one FMA: v * 2^32 + 1.5 * 2^52 has a unit in the last
// place of exactly 1, so the sum's low mantissa bits are round(v * 2^32) in
// two's complement, read off by subtracting the constant's bit pattern (no
// float-to-integer conversion instruction).  That needs |v| < 2^19 per
// contribution; particles whose values could approach it (|value| / h^2 >=
// 2^20, weights are below 0.36) raise LCB_DEVERR_FIXED_RANGE.  Sums have the
// range +-2^31.
constexpr double FIX_SCALE = 4294967296.0;            // 2^32
constexpr double FIX_INV = 1.0 / 4294967296.0;
constexpr double FIX_MAGIC = 6755399441055744.0;      // 1.5 * 2^52
constexpr double FIX_PARTICLE_LIMIT = 1048576.0;      // 2^20
typedef unsigned long long fix_t;

// round(v * 2^32) from fma(v, 2^32, FIX_MAGIC) (or any x = w * 2^32 * v + FIX_MAGIC)
__device__ __forceinline__ fix_t fix_bits(double x)
{
    return (fix_t)__double_as_longlong(x) - (fix_t)0x4338000000000000ull;
}

template <typename Acc>
__device__ __forceinline__ Acc to_acc(double v) { return Acc(v); }
template <>
__device__ __forceinline__ fix_t to_acc<fix_t>(double v)
{
    return fix_bits(fma(v, FIX_SCALE, FIX_MAGIC));
}

// Particles whose largest contribution could leave the fixed-point rounding
// range set the error word; nothing else changes.
template <typename Acc>
__device__ __forceinline__ void check_range(double, double, double, double, double, int *) {}
template <>
__device__ __forceinline__ void check_range<fix_t>(double dro, double djx, double djy, double djz,
                                                   double ih, int *err)
{
    const double m = fmax(fmax(fabs(dro), fabs(djx)), fmax(fabs(djy), fabs(djz))) * ih * ih;
    if (!(m < FIX_PARTICLE_LIMIT) && err) atomicOr(err, LCB_DEVERR_FIXED_RANGE);
}

template <typename Acc, int WX, int WY>
__device__ __forceinline__ void deposit_one(Acc *sw, Acc *gro, Acc *gjx, Acc *gjy, Acc *gjz,
                                            int N, double h, int wx0, int wy0, bool dep,
                                            int ix, int iy, double xl, double yl,
                                            double dro, double djx, double djy, double djz)
{
    constexpr int WSZ = WX * WY;
    if (!dep) return;
    double wx[5], wy[5];
    weights4(xl, wx);
    weights4(yl, wy);
    // w = (wx / h) (wy / h), with 1/h multiplications for the 30 quotients
    const double ih = 1.0 / h;
#pragma unroll
    for (int b = 0; b < 5; b++) wy[b] *= ih;
    const int lx = ix - 2 - wx0, ly = iy - 2 - wy0;
    const bool inwin = lx >= 0 && lx + 5 <= WX && ly >= 0 && ly + 5 <= WY;
#pragma unroll
    for (int a = 0; a < 5; a++) {
        const double wxa = wx[a] * ih;
#pragma unroll
        for (int b = 0; b < 5; b++) {
            const double w = wxa * wy[b];
            if (inwin) {
                const int c = (lx + a) * WY + ly + b;
                atomicAdd(sw + c, to_acc<Acc>(dro * w));
                atomicAdd(sw + WSZ + c, to_acc<Acc>(djx * w));
                atomicAdd(sw + 2 * WSZ + c, to_acc<Acc>(djy * w));
                atomicAdd(sw + 3 * WSZ + c, to_acc<Acc>(djz * w));
            } else {
                const int64_t c = (int64_t)(ix + a - 2) * N + iy + b - 2;
                atomicAdd(gro + c, to_acc<Acc>(dro * w));
                atomicAdd(gjx + c, to_acc<Acc>(djx * w));
                atomicAdd(gjy + c, to_acc<Acc>(djy * w));
                atomicAdd(gjz + c, to_acc<Acc>(djz * w));
            }
        }
    }
}

template <typename Acc>
__global__ void __launch_bounds__(DEP_THREADS)
k_deposit_tiled(int64_t n_per_sort, int Ns, int N, double h,
                const double *__restrict__ x_init, const double *__restrict__ y_init,
                const double *__restrict__ x_offt, const double *__restrict__ y_offt,
                const double *__restrict__ px_a, const double *__restrict__ py_a,
                const double *__restrict__ pz_a, const double *__restrict__ q_a,
                const double *__restrict__ m_a, Acc *ro, Acc *jx, Acc *jy, Acc *jz,
                int *err)
{
    static_assert(DEP_PPT == 2, "a thread owns two particles");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Acc *sw = reinterpret_cast<Acc *>(smem_raw);  // [4][WX][WY]
    constexpr int WSZ = DEP_WX * DEP_WY;
    const int s = blockIdx.z;
    const int64_t base = (int64_t)s * n_per_sort;
    const int half_n = N / 2;
    const int64_t NN = (int64_t)N * N;
    Acc *gro = ro + s * NN, *gjx = jx + s * NN, *gjy = jy + s * NN, *gjz = jz + s * NN;

    for (int t = threadIdx.x; t < 4 * WSZ; t += blockDim.x) sw[t] = Acc(0);
    // Tiles start on a lattice row whose cell also holds the next row, so
    // that a thread's two particles (slots t and t + DEP_THREADS: lattice
    // rows ti and ti + 1, ti even) usually share a cell; the grid has one
    // spare row of tiles for the shift.
    double dummy;
    int off = 0;
    if (Ns > 1 && cell_of(x_init[base] / h + 0.5, half_n, dummy) !=
                  cell_of(x_init[base + Ns] / h + 0.5, half_n, dummy))
        off = 1;
    const int i0 = blockIdx.y * DEP_TI - off, j0 = blockIdx.x * DEP_TJ;
    const int ir = i0 < 0 ? 0 : i0;
    if (ir >= Ns) return;
    // window origin from the tile's first particle's initial lattice position
    const int64_t k0 = base + (int64_t)ir * Ns + j0;
    const int wx0 = cell_of(x_init[k0] / h + 0.5, half_n, dummy) - 2 - DEP_SLACK;
    const int wy0 = cell_of(y_init[k0] / h + 0.5, half_n, dummy) - 2 - DEP_SLACK;
    // lattice spacing along x: two particles per cell?
    bool two = false;
    if (ir + 1 < Ns) {
        const double d = x_init[k0 + Ns] - x_init[k0];
        two = fabs(2 * d - h) < 0.25 * h;
    }
    __syncthreads();

    bool dep[2];
    double v[2][4], xl[2], yl[2];
    int ix[2], iy[2];
#pragma unroll
    for (int r = 0; r < DEP_PPT; r++) {
        int ti, tj;
        tile_slot(threadIdx.x + r * DEP_THREADS, two, ti, tj);
        const int i = i0 + ti, j = j0 + tj;
        dep[r] = i >= 0 && i < Ns && j < Ns;
        v[r][0] = v[r][1] = v[r][2] = v[r][3] = 0;
        xl[r] = yl[r] = 0;
        ix[r] = iy[r] = -1000;
        if (dep[r]) {
            const int64_t k = base + (int64_t)i * Ns + j;
            const double q = q_a[k];
            if (q == 0) {
                dep[r] = false;
            } else {
                const double m = m_a[k], px = px_a[k], py = py_a[k], pz = pz_a[k];
                const double gm = sqrt(m * m + px * px + py * py + pz * pz);
                const double ig = 1.0 / gm;
                const double dro = q / (1 - pz * ig);
                const double rg = dro * ig;
                v[r][0] = dro; v[r][1] = px * rg; v[r][2] = py * rg; v[r][3] = pz * rg;
                check_range<Acc>(v[r][0], v[r][1], v[r][2], v[r][3], 1.0 / h, err);
                ix[r] = cell_of((x_init[k] + x_offt[k]) / h + 0.5, half_n, xl[r]);
                iy[r] = cell_of((y_init[k] + y_offt[k]) / h + 0.5, half_n, yl[r]);
                if (!(ix[r] >= 2 && ix[r] < N - 2 && iy[r] >= 2 && iy[r] < N - 2)) {
                    if (err) atomicOr(err, LCB_DEVERR_PLASMA_STENCIL);
                    dep[r] = false;
                }
            }
        }
    }
    // FP64: two particles in one cell add their contributions before the
    // shared atomic (one atomic per stencil point and quantity for both)
    const int lx = ix[0] - 2 - wx0, ly = iy[0] - 2 - wy0;
    const bool joint = sizeof(Acc) == sizeof(double) && !std::is_integral<Acc>::value &&
                       dep[0] && dep[1] && ix[0] == ix[1] && iy[0] == iy[1] &&
                       lx >= 0 && lx + 5 <= DEP_WX && ly >= 0 && ly + 5 <= DEP_WY;
    if (joint) {
        double ax[5], ay[5], bx[5], by[5];
        weights4(xl[0], ax); weights4(yl[0], ay);
        weights4(xl[1], bx); weights4(yl[1], by);
        const double ih = 1.0 / h;
#pragma unroll
        for (int b = 0; b < 5; b++) { ay[b] *= ih; by[b] *= ih; }
#pragma unroll
        for (int a = 0; a < 5; a++) {
            const double xa = ax[a] * ih, xb = bx[a] * ih;
#pragma unroll
            for (int b = 0; b < 5; b++) {
                const double wa = xa * ay[b], wb = xb * by[b];
                const int c = (lx + a) * DEP_WY + ly + b;
#pragma unroll
                for (int q = 0; q < 4; q++)
                    atomicAdd(sw + q * WSZ + c, Acc(fma(v[0][q], wa, v[1][q] * wb)));
            }
        }
    } else {
#pragma unroll
        for (int r = 0; r < DEP_PPT; r++)
            deposit_one<Acc, DEP_WX, DEP_WY>(sw, gro, gjx, gjy, gjz, N, h, wx0, wy0, dep[r], ix[r],
                                              iy[r], xl[r], yl[r], v[r][0], v[r][1], v[r][2], v[r][3]);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < WSZ; t += blockDim.x) {
        const int gx = wx0 + t / DEP_WY, gy = wy0 + t % DEP_WY;
        if (gx < 0 || gx >= N || gy < 0 || gy >= N) continue;
        const int64_t c = (int64_t)gx * N + gy;
        const Acc v0 = sw[t], v1 = sw[WSZ + t], v2 = sw[2 * WSZ + t], v3 = sw[3 * WSZ + t];
        if (v0 != Acc(0)) atomicAdd(gro + c, v0);
        if (v1 != Acc(0)) atomicAdd(gjx + c, v1);
        if (v2 != Acc(0)) atomicAdd(gjy + c, v2);
        if (v3 != Acc(0)) atomicAdd(gjz + c, v3);
    }
}

template <typename T>
static size_t deposit_smem_bytes()
{
    return (size_t)4 * DEP_WX * DEP_WY * sizeof(T);
}

// ---------------------------------------------------------------------------
// Fused predictor-corrector stage: K2 (move_smart) followed by K3 (deposit)
// of the same particles, and for the first stage of an xi step K1 (the
// free-streaming estimate) in front (move.py:169-313, weights.py:151-190).
// A block owns a lattice tile of TI x TJ particles; the six field planes are
// staged in a shared-memory window around the tile for the midpoint gather,
// and the new position is deposited into a second window, flushed with
// global atomics; particles whose stencil leaves a window use global memory.
// FP64 (FT = double): each particle's gather and push are those of K2 and
// K3 (same quotients, same summation order); the deposit sums the two
// particles of a cell before the shared atomic.  Mixed precision
// (FT = float): coordinates and momenta stay FP64; the gather reads an FP32
// copy of the field window with FP32 weights (the planes come from the FP32
// field solve); the deposit keeps FP64 weights, scales each particle's four
// values by 2^32 / h^2 once, and rounds every contribution to a 64-bit
// integer with one FMA against FIX_MAGIC, summed with integer atomics.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void weights4f(float x, float w[5])
{
    const float x2 = x * x, x3 = x2 * x, x4 = x3 * x;
    const float a = 0.5f - x, b = 0.5f + x;
    const float r6 = 1.0f / 6.0f, r24 = 1.0f / 24.0f;
    w[0] = a * a * a * a * r24;
    w[1] = 19 / 96.f - 11 / 24.f * x + x2 * 0.25f + x3 * r6 - x4 * r6;
    w[2] = 115 / 192.f - 5 / 8.f * x2 + x4 * 0.25f;
    w[3] = 19 / 96.f + 11 / 24.f * x + x2 * 0.25f - x3 * r6 - x4 * r6;
    w[4] = b * b * b * b * r24;
}

__device__ __forceinline__ void weights_of(float x, float w[5]) { weights4f(x, w); }
__device__ __forceinline__ void weights_of(double x, double w[5]) { weights4(x, w); }

// The five weights of a particle whose cell is s (0 or 1) cells past the
// origin of a six-point footprint, as six weights (zero outside).
template <typename W>
__device__ __forceinline__ void shift6(const W w[5], int s, W o[6])
{
#pragma unroll
    for (int k = 0; k < 6; k++) {
        const W keep = k < 5 ? w[k] : W(0), moved = k > 0 ? w[k - 1] : W(0);
        o[k] = s ? moved : keep;
    }
}

// Packed FP32 pairs (sm_100 f32x2 arithmetic): two floats in one 64-bit
// register pair, and an FMA on both lanes.
__device__ __forceinline__ unsigned long long f32x2(float lo, float hi)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void unpack_f32x2(unsigned long long v, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long fma_f32x2(unsigned long long a, unsigned long long b,
                                                        unsigned long long c)
{
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// Field window in shared memory: the six field values of a cell are stored
// together, so that one stencil point of the gather takes vector loads
// (FP32: a float4 of Ex, Ey, Ez, Bx and a float2 of By, Bz; FP64: three
// double2) instead of six scalar ones.  A quarter warp reads eight
// consecutive cells of a row (128 contiguous bytes per load), so rows need
// no padding.
template <typename FT> struct FieldWin;
template <> struct FieldWin<float> {
    static constexpr int bytes_per_cell = 24;
    __device__ static void put(unsigned char *w, int ncell, int c, const float v[6])
    {
        reinterpret_cast<float4 *>(w)[c] = make_float4(v[0], v[1], v[2], v[3]);
        reinterpret_cast<float2 *>(w + 16 * ncell)[c] = make_float2(v[4], v[5]);
    }
    __device__ static void get(const unsigned char *w, int ncell, int c, float v[6])
    {
        const float4 a = reinterpret_cast<const float4 *>(w)[c];
        const float2 b = reinterpret_cast<const float2 *>(w + 16 * ncell)[c];
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y;
    }
};
template <> struct FieldWin<double> {
    static constexpr int bytes_per_cell = 48;
    __device__ static void put(unsigned char *w, int ncell, int c, const double v[6])
    {
        double2 *d = reinterpret_cast<double2 *>(w);
        d[c] = make_double2(v[0], v[1]);
        d[ncell + c] = make_double2(v[2], v[3]);
        d[2 * ncell + c] = make_double2(v[4], v[5]);
    }
    __device__ static void get(const unsigned char *w, int ncell, int c, double v[6])
    {
        const double2 *d = reinterpret_cast<const double2 *>(w);
        const double2 a = d[c], b = d[ncell + c], e = d[2 * ncell + c];
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y; v[4] = e.x; v[5] = e.y;
    }
};

// Midpoint gather of one particle from the window when the stencil fits in
// it, else from the FP64 planes in HBM; weights and sums in FT.
template <typename FT, int WX, int WY>
__device__ __forceinline__ void gather_one(const unsigned char *sf, const double *const *fld, int N,
                                           int wx0, int wy0, int ix, int iy, FT xl, FT yl,
                                           FT F[6])
{
    FT wx[5], wy[5];
    weights_of(xl, wx);
    weights_of(yl, wy);
    const int lx = ix - 2 - wx0, ly = iy - 2 - wy0;
    if (lx >= 0 && lx + 5 <= WX && ly >= 0 && ly + 5 <= WY) {
#pragma unroll
        for (int a = 0; a < 5; a++) {
#pragma unroll
            for (int b = 0; b < 5; b++) {
                const FT w = wx[a] * wy[b];
                FT v[6];
                FieldWin<FT>::get(sf, WX * WY, (lx + a) * WY + ly + b, v);
#pragma unroll
                for (int f = 0; f < 6; f++) F[f] += v[f] * w;
            }
        }
    } else {
#pragma unroll 1
        for (int a = 0; a < 5; a++) {
            const int row = (ix + a - 2) * N + iy - 2;
#pragma unroll
            for (int b = 0; b < 5; b++) {
                const FT w = wx[a] * wy[b];
#pragma unroll
                for (int f = 0; f < 6; f++) F[f] += (FT)__ldg(fld[f] + row + b) * w;
            }
        }
    }
}

// The shared-memory window keeps each fixed-point sum as two 32-bit words,
// because 32-bit integer atomics are native in shared memory and 64-bit ones
// are not: a contribution c (in units of 2^-32) adds its low 20 bits to an
// unsigned word and c >> 20 to a signed word; the flush recombines
// (hi << 20) + lo exactly.  A block adds at most 2 x 256 contributions to a
// cell, so the low word stays below 2^29 and, with |c| < 2^41 (particles
// whose scaled values reach 2^42, i.e. |value| / h^2 >= 1024, take the
// global 64-bit path instead), the high word below 2^30.
constexpr double FIX_SHARED_LIMIT = 4398046511104.0;   // 2^42, on values scaled by 2^32 / h^2

// t = FIX_MAGIC + c exactly (the rounding FMA's result).  FIX_MAGIC's low
// word is zero, so the low word of t's bit pattern is c mod 2^32 and its high
// word minus 0x43380000 is floor(c / 2^32); c >> 20 is then one funnel shift.
__device__ __forceinline__ void shared_fix_add(unsigned *lo, int *hi, int idx, double t)
{
    const unsigned w0 = (unsigned)__double2loint(t);
    const unsigned w1 = (unsigned)(__double2hiint(t) - 0x43380000);
    atomicAdd(lo + idx, w0 & 0xFFFFFu);
    atomicAdd(hi + idx, (int)__funnelshift_r(w0, w1, 20));
}

__device__ __forceinline__ bool shared_fix_ok(const double sv[4])
{
    return fmax(fmax(fabs(sv[0]), fabs(sv[1])), fmax(fabs(sv[2]), fabs(sv[3]))) < FIX_SHARED_LIMIT;
}

// Deposit of one particle's scaled values (FP64 weights, fixed-point sums).
template <int WX, int WY>
__device__ __forceinline__ void deposit_fix_one(unsigned *swl, int *swh, fix_t *const *g, int N,
                                                int wx0, int wy0, int cx, int cy, double xl,
                                                double yl, const double sv[4])
{
    constexpr int WSZ = WX * WY;
    double wx[5], wy[5];
    weights4(xl, wx);
    weights4(yl, wy);
    const int lx = cx - 2 - wx0, ly = cy - 2 - wy0;
    if (lx >= 0 && lx + 5 <= WX && ly >= 0 && ly + 5 <= WY && shared_fix_ok(sv)) {
#pragma unroll
        for (int a = 0; a < 5; a++) {
#pragma unroll
            for (int b = 0; b < 5; b++) {
                const double w = wx[a] * wy[b];
                const int c = (lx + a) * WY + ly + b;
#pragma unroll
                for (int q = 0; q < 4; q++)
                    shared_fix_add(swl, swh, q * WSZ + c, fma(sv[q], w, FIX_MAGIC));
            }
        }
    } else {
#pragma unroll 1
        for (int a = 0; a < 5; a++) {
#pragma unroll
            for (int b = 0; b < 5; b++) {
                const double w = wx[a] * wy[b];
                const int64_t c = (int64_t)(cx + a - 2) * N + cy + b - 2;
#pragma unroll
                for (int q = 0; q < 4; q++)
                    atomicAdd(g[q] + c, fix_bits(fma(sv[q], w, FIX_MAGIC)));
            }
        }
    }
}

// FP64 deposit window: every contribution v (an FP64 value in the units of
// the output currents) is rounded to a multiple of 2^-56 and summed as an
// integer split over three 32-bit words -- bits 0-19 and 20-39 unsigned,
// bits 40 up signed -- with 32-bit shared integer atomics, which run the
// fused stage about 7% faster than FP64 shared atomics.  A particle whose
// contributions could reach |v| = 2^4 (weights wx wy are below 0.36)
// deposits into HBM with FP64 atomics instead, so |v| 2^56 <
// 2^60 and, with at most 2 x 256 contributions per cell and block (every
// particle of the block at most once), no word overflows.  The integer sums
// are exact and independent of the order of the atomics; each contribution
// differs from FP64 by at most 2^-57, and the flush recombines the words
// with one FP64 rounding before adding the value to the outputs.  The
// particle's values arrive multiplied by 2^56 (exact: a power of two), so a
// contribution's integer is one rounding conversion of its product.
constexpr double FIX56_SCALE = 72057594037927936.0;   // 2^56
constexpr double FIX56_LIMIT = 16.0 * FIX56_SCALE;    // per contribution, in the window

// v: a contribution in units of 2^-56
__device__ __forceinline__ void fix56_add(unsigned *w0, unsigned *w1, int *w2, int idx, double v)
{
    const long long c = __double2ll_rn(v);
    atomicAdd(w0 + idx, (unsigned)c & 0xFFFFFu);
    atomicAdd(w1 + idx, (unsigned)(c >> 20) & 0xFFFFFu);
    atomicAdd(w2 + idx, (int)(c >> 40));
}

__device__ __forceinline__ double fix56_value(unsigned w0, unsigned w1, int w2)
{
    return ((double)w2 * 1099511627776.0 + (double)w1 * 1048576.0 + (double)w0) * (1.0 / FIX56_SCALE);
}

// One particle's FP64 deposit (weights.py:151-190 arithmetic, w = (wx / h)
// (wy / h)) into the three-word window, or into HBM with FP64 atomics when
// the stencil leaves the window or a contribution could leave the range;
// sv: the particle's values in units of 2^-56.
template <int WX, int WY>
__device__ __forceinline__ void deposit_fix56_one(unsigned *w0, unsigned *w1, int *w2, double *const *g,
                                                  int N, double ih, int wx0, int wy0, int cx, int cy,
                                                  double xl, double yl, const double sv[4])
{
    constexpr int WSZ = WX * WY;
    double wx[5], wy[5];
    weights4(xl, wx);
    weights4(yl, wy);
#pragma unroll
    for (int b = 0; b < 5; b++) wy[b] *= ih;
    const int lx = cx - 2 - wx0, ly = cy - 2 - wy0;
    const double m = fmax(fmax(fabs(sv[0]), fabs(sv[1])), fmax(fabs(sv[2]), fabs(sv[3])));
    const bool inwin = lx >= 0 && lx + 5 <= WX && ly >= 0 && ly + 5 <= WY &&
                       m * (0.36 * ih * ih) < FIX56_LIMIT;
#pragma unroll
    for (int a = 0; a < 5; a++) {
        const double wxa = wx[a] * ih;
#pragma unroll
        for (int b = 0; b < 5; b++) {
            const double w = wxa * wy[b];
            if (inwin) {
                const int c = (lx + a) * WY + ly + b;
#pragma unroll
                for (int q = 0; q < 4; q++) fix56_add(w0, w1, w2, q * WSZ + c, sv[q] * w);
            } else {
                const int64_t c = (int64_t)(cx + a - 2) * N + cy + b - 2;
#pragma unroll
                for (int q = 0; q < 4; q++) atomicAdd(g[q] + c, sv[q] * w * (1.0 / FIX56_SCALE));
            }
        }
    }
}

// A thread owns two particles, lattice slots t and t + DEP_THREADS, which on
// the 2 x 2 per cell lattice are the two lattice rows of one cell.  While
// both sit in the same cell the window values of the gather are loaded once
// for the two, and their deposits are added before the shared atomics (each
// contribution is still rounded on its own: fma(sA, wA, fma(sB, wB, M)) adds
// two integers), which halves the shared-memory traffic of both phases.
template <typename FT> struct StageAcc;
template <> struct StageAcc<float> { typedef fix_t type; };
template <> struct StageAcc<double> { typedef double type; };

template <typename FT, int WX, int WY, bool FIRST>
__global__ void __launch_bounds__(DEP_THREADS, sizeof(FT) == 4 ? 3 : 2)
k_move_deposit_pair(int64_t n_per_sort, int Ns, int N, double h, double xi_step, double boundary,
                  const double *__restrict__ Exf, const double *__restrict__ Eyf,
                  const double *__restrict__ Ezf, const double *__restrict__ Bxf,
                  const double *__restrict__ Byf, const double *__restrict__ Bzf,
                  const double *__restrict__ x_init, const double *__restrict__ y_init,
                  const double *__restrict__ xo_p, const double *__restrict__ yo_p,
                  const double *__restrict__ px_p, const double *__restrict__ py_p,
                  const double *__restrict__ pz_p, const double *__restrict__ q_p,
                  const double *__restrict__ m_a,
                  double *q_f, double *xo_f, double *yo_f, double *px_f, double *py_f,
                  double *pz_f, typename StageAcc<FT>::type *ro, typename StageAcc<FT>::type *jx,
                  typename StageAcc<FT>::type *jy, typename StageAcc<FT>::type *jz, int *err)
{
    // launched after its predecessor's tail (programmatic launch): no global
    // memory access before the wait
    pdl_wait();
    pdl_trigger();
    constexpr bool MIXED = sizeof(FT) == 4;
    typedef typename StageAcc<FT>::type Acc;
    static_assert(DEP_PPT == 2, "a thread owns two particles");
    constexpr int WSZ = WX * WY;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // deposit window: mixed, [4][WX][WY] low and high words of the 2^-32
    // fixed-point sums; FP64, three words per sum of the 2^-56 ones
    constexpr int DEP_WORDS = MIXED ? 2 : 3;
    unsigned *swl = reinterpret_cast<unsigned *>(smem_raw);    // [4][WX][WY] word 0
    int *swh = reinterpret_cast<int *>(swl + 4 * WSZ);         // mixed: high words
    unsigned *sw1 = swl + 4 * WSZ;                             // FP64: words 1 and 2
    int *sw2 = reinterpret_cast<int *>(swl + 8 * WSZ);
    unsigned char *sf = smem_raw + (size_t)DEP_WORDS * 4 * WSZ * 4;  // fields, FieldWin
    const int s = blockIdx.z;
    const int64_t base = (int64_t)s * n_per_sort;
    const int half_n = N / 2;
    const int64_t NN = (int64_t)N * N;
    Acc *const g4[4] = {ro + s * NN, jx + s * NN, jy + s * NN, jz + s * NN};
    const double *const fld[6] = {Exf, Eyf, Ezf, Bxf, Byf, Bzf};
    const double ih = 1.0 / h;

    // Tiles start on a lattice row whose cell also holds the next row, so
    // that a thread's two rows (ti, ti + 1 with ti even) share a cell: when
    // rows 0 and 1 sit in different cells the tiles are shifted up by one
    // row (the grid has one spare row of tiles for it).  The tile's first
    // particle is read for both possible shifts at once, so that the tile
    // origin costs one round trip to memory.
    double dummy;
    const int ia = blockIdx.y * DEP_TI, ib = ia > 0 ? ia - 1 : 0;   // tile row for off = 0, 1
    const int64_t ka = base + (int64_t)(ia < Ns ? ia : 0) * Ns + blockIdx.x * DEP_TJ;
    const int64_t kb = base + (int64_t)ib * Ns + blockIdx.x * DEP_TJ;
    const bool two_rows = Ns > 1;
    const double r0x = x_init[base], r1x = two_rows ? x_init[base + Ns] : r0x;
    const double xa = x_init[ka], ya = y_init[ka], xb = x_init[kb], yb = y_init[kb];
    const double xa1 = ia + 1 < Ns ? x_init[ka + Ns] : xa, xb1 = ib + 1 < Ns ? x_init[kb + Ns] : xb;
    const int off = (two_rows && cell_of(r0x / h + 0.5, half_n, dummy) !=
                                 cell_of(r1x / h + 0.5, half_n, dummy)) ? 1 : 0;
    const int i0 = blockIdx.y * DEP_TI - off, j0 = blockIdx.x * DEP_TJ;
    const int ir = i0 < 0 ? 0 : i0;
    if (ir >= Ns) return;
    const int64_t k0 = base + (int64_t)ir * Ns + j0;
    const double x0 = off ? xb : xa, y0 = off ? yb : ya, x1 = off ? xb1 : xa1;
    const int wx0 = cell_of(x0 / h + 0.5, half_n, dummy) - 2 - DEP_SLACK;
    const int wy0 = cell_of(y0 / h + 0.5, half_n, dummy) - 2 - DEP_SLACK;
    bool two = false;
    if (ir + 1 < Ns) {
        const double d = x1 - x0;
        two = fabs(2 * d - h) < 0.25 * h;
    }
    (void)k0;

    // ---- the particles' first loads, issued before the window fill ----
    int64_t kk[2];
    bool live[2], zero_p[2];
    double L_xo0[2], L_yo0[2], L_xi[2], L_yi[2], L_q[2], L_xof[2], L_yof[2];
    double L_m[2], L_px[2], L_py[2], L_pz[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
        int ti, tj;
        tile_slot(threadIdx.x + p * DEP_THREADS, two, ti, tj);
        const int i = i0 + ti, j = j0 + tj;
        live[p] = i >= 0 && i < Ns && j < Ns;
        kk[p] = base + (int64_t)i * Ns + j;
        L_xo0[p] = L_yo0[p] = L_xi[p] = L_yi[p] = L_q[p] = L_xof[p] = L_yof[p] = 0;
        L_m[p] = L_px[p] = L_py[p] = L_pz[p] = 0;
        if (!live[p]) continue;
        const int64_t k = kk[p];
        L_xo0[p] = xo_p[k]; L_yo0[p] = yo_p[k];
        L_xi[p] = x_init[k]; L_yi[p] = y_init[k];
        if (FIRST) {
            L_m[p] = m_a[k]; L_px[p] = px_p[k]; L_py[p] = py_p[k]; L_pz[p] = pz_p[k];
            L_q[p] = q_p[k];
        } else {
            L_q[p] = q_f[k]; L_xof[p] = xo_f[k]; L_yof[p] = yo_f[k];
        }
    }

    for (int t = threadIdx.x; t < DEP_WORDS * 4 * WSZ; t += blockDim.x) swl[t] = 0u;
    // the field window, FILL_BATCH cells per thread at a time: the batch's
    // loads are all in flight before the first store to the window
    constexpr int FILL_ITERS = (WSZ + DEP_THREADS - 1) / DEP_THREADS, FILL_BATCH = 3;
#pragma unroll
    for (int k0 = 0; k0 < FILL_ITERS; k0 += FILL_BATCH) {
        FT v[FILL_BATCH][6];
#pragma unroll
        for (int k = 0; k < FILL_BATCH; k++) {
            const int t = threadIdx.x + (k0 + k) * DEP_THREADS;
            const int gx = wx0 + t / WY, gy = wy0 + t % WY;
            const bool in = k0 + k < FILL_ITERS && t < WSZ && gx >= 0 && gx < N && gy >= 0 && gy < N;
            const int64_t g = (int64_t)gx * N + gy;
#pragma unroll
            for (int f = 0; f < 6; f++) v[k][f] = in ? (FT)__ldg(fld[f] + g) : FT(0);
        }
#pragma unroll
        for (int k = 0; k < FILL_BATCH; k++) {
            const int t = threadIdx.x + (k0 + k) * DEP_THREADS;
            if (k0 + k < FILL_ITERS && t < WSZ) FieldWin<FT>::put(sf, WSZ, t, v[k]);
        }
    }
    __syncthreads();

    // ---- phase 1: K1 (first stage) and the midpoint of each particle ----
    int ix[2], iy[2];
    FT xlf[2], ylf[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
        zero_p[p] = false;
        ix[p] = iy[p] = -1000;
        xlf[p] = ylf[p] = FT(0);
        if (!live[p]) continue;
        const int64_t k = kk[p];
        const double xo0 = L_xo0[p], yo0 = L_yo0[p];
        const double qk = L_q[p];
        double xof, yof;
        if (FIRST) {
            const double mk = L_m[p], opx = L_px[p], opy = L_py[p], opz = L_pz[p];
            xof = xo0; yof = yo0;
            if (mk != 0) {
                const double gm = sqrt(mk * mk + opz * opz + opx * opx + opy * opy);
                const double adv = xi_step / (gm - opz);
                xof += opx * adv;
                yof += opy * adv;
            }
            if (qk == 0) {
                xo_f[k] = xof; yo_f[k] = yof;
                px_f[k] = opx; py_f[k] = opy; pz_f[k] = opz;
                q_f[k] = qk;
            }
        } else {
            xof = L_xof[p]; yof = L_yof[p];
        }
        if (qk == 0) { live[p] = false; continue; }
        double xh = L_xi[p] + (xo0 + xof) / 2;
        double yh = L_yi[p] + (yo0 + yof) / 2;
        bool z = false;
        if (xh > boundary)  { xh =  2 * boundary - xh; z = true; }
        if (xh < -boundary) { xh = -2 * boundary - xh; z = true; }
        if (yh > boundary)  { yh =  2 * boundary - yh; z = true; }
        if (yh < -boundary) { yh = -2 * boundary - yh; z = true; }
        zero_p[p] = z;
        double xl, yl;
        // FP64: the quotient of K2 itself; mixed: the reciprocal
        ix[p] = cell_of(xh * ih + 0.5, half_n, xl);
        iy[p] = cell_of(yh * ih + 0.5, half_n, yl);
        xlf[p] = (FT)xl; ylf[p] = (FT)yl;
        if (!(ix[p] >= 2 && ix[p] < N - 2 && iy[p] >= 2 && iy[p] < N - 2)) {
            if (err) atomicOr(err, LCB_DEVERR_PLASMA_STENCIL);
            ix[p] = -1000;  // no gather: zero fields, as in the reference's skip
        }
        // the push's mass and momenta, loaded while the gather runs
        if (!FIRST) { L_m[p] = m_a[k]; L_px[p] = px_p[k]; L_py[p] = py_p[k]; L_pz[p] = pz_p[k]; }
    }

    // ---- phase 2: gather ----
    // Three forms, chosen per warp so that a warp runs one of them: when
    // every lane's two particles share a cell (or the lane has none), the
    // 5 x 5 joint form; otherwise lanes whose particles sit in neighbouring
    // cells gather both over one 6 x 6 footprint (each particle's weights
    // zero outside its own 5 x 5), and the rest one particle at a time.  The
    // zero-weight terms leave each particle's sums unchanged.
    FT F0[6] = {0, 0, 0, 0, 0, 0}, F1[6] = {0, 0, 0, 0, 0, 0};
    {
        const int lx = ix[0] - 2 - wx0, ly = iy[0] - 2 - wy0;
        const bool joint = ix[0] >= 0 && ix[0] == ix[1] && iy[0] == iy[1] &&
                           lx >= 0 && lx + 5 <= WX && ly >= 0 && ly + 5 <= WY;
        const int mx = min(ix[0], ix[1]), my = min(iy[0], iy[1]);
        const int px0 = mx - 2 - wx0, py0 = my - 2 - wy0;
        const bool pair = ix[0] >= 0 && ix[1] >= 0 && abs(ix[1] - ix[0]) <= 1 &&
                          abs(iy[1] - iy[0]) <= 1 && px0 >= 0 && px0 + 6 <= WX &&
                          py0 >= 0 && py0 + 6 <= WY;
        const bool idle = ix[0] < 0 && ix[1] < 0;
        if (!__all_sync(0xffffffffu, joint || idle)) {
            if (pair && MIXED) {
                float ax[6], ay[6], bx[6], by[6], t[5];
                weights4f((float)xlf[0], t); shift6(t, ix[0] - mx, ax);
                weights4f((float)ylf[0], t); shift6(t, iy[0] - my, ay);
                weights4f((float)xlf[1], t); shift6(t, ix[1] - mx, bx);
                weights4f((float)ylf[1], t); shift6(t, iy[1] - my, by);
                unsigned long long A[3] = {0ull, 0ull, 0ull}, B[3] = {0ull, 0ull, 0ull};
#pragma unroll
                for (int a = 0; a < 6; a++) {
#pragma unroll
                    for (int b = 0; b < 6; b++) {
                        const float wa = ax[a] * ay[b], wb = bx[a] * by[b];
                        const unsigned long long wa2 = f32x2(wa, wa), wb2 = f32x2(wb, wb);
                        const int c = (px0 + a) * WY + py0 + b;
                        const float4 p = reinterpret_cast<const float4 *>(sf)[c];
                        const float2 q = reinterpret_cast<const float2 *>(sf + 16 * WSZ)[c];
                        const unsigned long long v3[3] = {f32x2(p.x, p.y), f32x2(p.z, p.w),
                                                          f32x2(q.x, q.y)};
#pragma unroll
                        for (int k = 0; k < 3; k++) {
                            A[k] = fma_f32x2(v3[k], wa2, A[k]);
                            B[k] = fma_f32x2(v3[k], wb2, B[k]);
                        }
                    }
                }
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    float lo, hi;
                    unpack_f32x2(A[k], lo, hi); F0[2 * k] = (FT)lo; F0[2 * k + 1] = (FT)hi;
                    unpack_f32x2(B[k], lo, hi); F1[2 * k] = (FT)lo; F1[2 * k + 1] = (FT)hi;
                }
            } else if (pair) {
                FT ax[6], ay[6], bx[6], by[6], t[5];
                weights_of(xlf[0], t); shift6(t, ix[0] - mx, ax);
                weights_of(ylf[0], t); shift6(t, iy[0] - my, ay);
                weights_of(xlf[1], t); shift6(t, ix[1] - mx, bx);
                weights_of(ylf[1], t); shift6(t, iy[1] - my, by);
#pragma unroll
                for (int a = 0; a < 6; a++) {
#pragma unroll
                    for (int b = 0; b < 6; b++) {
                        const FT wa = ax[a] * ay[b], wb = bx[a] * by[b];
                        FT v[6];
                        FieldWin<FT>::get(sf, WSZ, (px0 + a) * WY + py0 + b, v);
#pragma unroll
                        for (int f = 0; f < 6; f++) {
                            F0[f] += v[f] * wa;
                            F1[f] += v[f] * wb;
                        }
                    }
                }
            } else {
                if (ix[0] >= 0)
                    gather_one<FT, WX, WY>(sf, fld, N, wx0, wy0, ix[0], iy[0], xlf[0], ylf[0], F0);
                if (ix[1] >= 0)
                    gather_one<FT, WX, WY>(sf, fld, N, wx0, wy0, ix[1], iy[1], xlf[1], ylf[1], F1);
            }
        } else if (joint && MIXED) {
            // FP32: the window's float4 / float2 of a cell are register pairs
            // (Ex Ey)(Ez Bx)(By Bz), accumulated with packed f32x2 FMAs
            // (per lane the same rounding as the scalar FMAs)
            float ax[5], ay[5], bx[5], by[5];
            weights4f((float)xlf[0], ax); weights4f((float)ylf[0], ay);
            weights4f((float)xlf[1], bx); weights4f((float)ylf[1], by);
            unsigned long long A[3] = {0ull, 0ull, 0ull}, B[3] = {0ull, 0ull, 0ull};
            // stencil rows in a rolled loop, as in the deposit
            int row = lx * WY + ly;
#pragma unroll 1
            for (int a = 0; a < 5; a++) {
#pragma unroll
                for (int b = 0; b < 5; b++) {
                    const float wa = ax[0] * ay[b], wb = bx[0] * by[b];
                    const unsigned long long wa2 = f32x2(wa, wa), wb2 = f32x2(wb, wb);
                    const int c = row + b;
                    const float4 p = reinterpret_cast<const float4 *>(sf)[c];
                    const float2 q = reinterpret_cast<const float2 *>(sf + 16 * WSZ)[c];
                    const unsigned long long v3[3] = {f32x2(p.x, p.y), f32x2(p.z, p.w), f32x2(q.x, q.y)};
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        A[k] = fma_f32x2(v3[k], wa2, A[k]);
                        B[k] = fma_f32x2(v3[k], wb2, B[k]);
                    }
                }
#pragma unroll
                for (int k = 0; k < 4; k++) { ax[k] = ax[k + 1]; bx[k] = bx[k + 1]; }
                row += WY;
            }
#pragma unroll
            for (int k = 0; k < 3; k++) {
                float lo, hi;
                unpack_f32x2(A[k], lo, hi); F0[2 * k] = (FT)lo; F0[2 * k + 1] = (FT)hi;
                unpack_f32x2(B[k], lo, hi); F1[2 * k] = (FT)lo; F1[2 * k + 1] = (FT)hi;
            }
        } else if (joint) {
            FT ax[5], ay[5], bx[5], by[5];
            weights_of(xlf[0], ax); weights_of(ylf[0], ay);
            weights_of(xlf[1], bx); weights_of(ylf[1], by);
            int row = lx * WY + ly;
#pragma unroll 1
            for (int a = 0; a < 5; a++) {
#pragma unroll
                for (int b = 0; b < 5; b++) {
                    const FT wa = ax[0] * ay[b], wb = bx[0] * by[b];
                    FT v[6];
                    FieldWin<FT>::get(sf, WSZ, row + b, v);
#pragma unroll
                    for (int f = 0; f < 6; f++) {
                        F0[f] += v[f] * wa;
                        F1[f] += v[f] * wb;
                    }
                }
#pragma unroll
                for (int k = 0; k < 4; k++) { ax[k] = ax[k + 1]; bx[k] = bx[k + 1]; }
                row += WY;
            }
        }
    }

    // ---- phase 3: push (FP64) and the deposit values ----
    double sv[2][4];
    int cx[2], cy[2];
    double dxl[2], dyl[2];
#pragma unroll
    for (int p = 0; p < 2; p++) {
        cx[p] = -1000; cy[p] = 0; dxl[p] = dyl[p] = 0;
        sv[p][0] = sv[p][1] = sv[p][2] = sv[p][3] = 0;
        if (!live[p]) continue;
        const int64_t k = kk[p];
        const FT *Fp = p ? F1 : F0;
        const double Ex = Fp[0], Ey = Fp[1], Ez = Fp[2], Bx = Fp[3], By = Fp[4], Bz = Fp[5];
        const double mk = L_m[p], qk = L_q[p];
        const double opx = L_px[p], opy = L_py[p], opz = L_pz[p];
        const double xi0 = x_init[k], yi0 = y_init[k];
        double px = opx, py = opy, pz = opz;
        if (zero_p[p]) px = py = pz = 0;
        double gm, dpx, dpy, dpz;
#pragma unroll
        for (int it = 0; it < 2; it++) {
            gm = sqrt(mk * mk + px * px + py * py + pz * pz);
            // f (E + v x B) with v = p / gm and f = q dxi / (1 - vz), as
            // q dxi (gm E + p x B) / (gm - pz): one quotient (algebraically
            // the reference's two, move.py:234-239)
            const double r = qk * xi_step / (gm - pz);
            dpx = r * (gm * Ex + py * Bz - pz * By);
            dpy = r * (gm * Ey - px * Bz + pz * Bx);
            dpz = r * (gm * Ez + px * By - py * Bx);
            px = opx + dpx * 0.5; py = opy + dpy * 0.5; pz = opz + dpz * 0.5;
        }
        gm = sqrt(mk * mk + px * px + py * py + pz * pz);
        const double adv = xi_step / (gm - pz);
        double xo = xo_p[k] + px * adv;
        double yo = yo_p[k] + py * adv;
        px = opx + dpx; py = opy + dpy; pz = opz + dpz;
        double x = xi0 + xo, y = yi0 + yo;
        if (x > boundary)  { x =  2 * boundary - x; xo = x - xi0; px = py = pz = 0; }
        if (x < -boundary) { x = -2 * boundary - x; xo = x - xi0; px = py = pz = 0; }
        if (y > boundary)  { y =  2 * boundary - y; yo = y - yi0; px = py = pz = 0; }
        if (y < -boundary) { y = -2 * boundary - y; yo = y - yi0; px = py = pz = 0; }
        bool absorbed = false;
        if (x >= boundary || x <= -boundary || y >= boundary || y <= -boundary) {
            xo = yo = 0; px = py = pz = 0;
            absorbed = true;
        }
        xo_f[k] = xo; yo_f[k] = yo;
        px_f[k] = px; py_f[k] = py; pz_f[k] = pz;
        if (FIRST || absorbed) q_f[k] = absorbed ? 0.0 : qk;
        if (absorbed) continue;
        const double gd = sqrt(mk * mk + px * px + py * py + pz * pz);
        // q / (1 - pz / gd) and p q / (gd - pz): one quotient (weights.py:
        // 164-168 has two)
        const double r = qk / (gd - pz);
        const double dro = r * gd, djx = r * px, djy = r * py, djz = r * pz;
        if (MIXED) check_range<fix_t>(dro, djx, djy, djz, ih, err);
        const int c_x = cell_of((xi0 + xo) * ih + 0.5, half_n, dxl[p]);
        const int c_y = cell_of((yi0 + yo) * ih + 0.5, half_n, dyl[p]);
        if (!(c_x >= 2 && c_x < N - 2 && c_y >= 2 && c_y < N - 2)) {
            if (err) atomicOr(err, LCB_DEVERR_PLASMA_STENCIL);
            continue;
        }
        cx[p] = c_x; cy[p] = c_y;
        // values in fixed-point units: mixed, 2^32 (with the 1/h^2 of the
        // weights); FP64, 2^56
        const double sc = MIXED ? FIX_SCALE * ih * ih : FIX56_SCALE;
        sv[p][0] = dro * sc; sv[p][1] = djx * sc; sv[p][2] = djy * sc; sv[p][3] = djz * sc;
    }

    // ---- phase 4: deposit ----
    // The gather's three forms again (warp-uniform choice), on the new cells.
    const int mcx = min(cx[0], cx[1]), mcy = min(cy[0], cy[1]);
    const int dx0 = mcx - 2 - wx0, dy0 = mcy - 2 - wy0;
    const bool dpair = cx[0] >= 0 && cx[1] >= 0 && abs(cx[1] - cx[0]) <= 1 &&
                       abs(cy[1] - cy[0]) <= 1 && dx0 >= 0 && dx0 + 6 <= WX && dy0 >= 0 &&
                       dy0 + 6 <= WY;
    const bool didle = cx[0] < 0 && cx[1] < 0;
    if constexpr (MIXED) {
        {
            const int lx = cx[0] - 2 - wx0, ly = cy[0] - 2 - wy0;
            const bool ok = shared_fix_ok(sv[0]) && shared_fix_ok(sv[1]);
            const bool joint = cx[0] >= 0 && cx[0] == cx[1] && cy[0] == cy[1] &&
                               lx >= 0 && lx + 5 <= WX && ly >= 0 && ly + 5 <= WY && ok;
            if (!__all_sync(0xffffffffu, joint || didle)) {
                if (dpair && ok) {
                    double ax[6], ay[6], bx[6], by[6], t[5];
                    weights4(dxl[0], t); shift6(t, cx[0] - mcx, ax);
                    weights4(dyl[0], t); shift6(t, cy[0] - mcy, ay);
                    weights4(dxl[1], t); shift6(t, cx[1] - mcx, bx);
                    weights4(dyl[1], t); shift6(t, cy[1] - mcy, by);
                    int row = dx0 * WY + dy0;
#pragma unroll 1
                    for (int a = 0; a < 6; a++) {
#pragma unroll
                        for (int b = 0; b < 6; b++) {
                            const double wa = ax[0] * ay[b], wb = bx[0] * by[b];
#pragma unroll
                            for (int q = 0; q < 4; q++)
                                shared_fix_add(swl, swh, q * WSZ + row + b,
                                               fma(sv[0][q], wa, fma(sv[1][q], wb, FIX_MAGIC)));
                        }
#pragma unroll
                        for (int k = 0; k < 5; k++) { ax[k] = ax[k + 1]; bx[k] = bx[k + 1]; }
                        row += WY;
                    }
                } else {
                    if (cx[0] >= 0)
                        deposit_fix_one<WX, WY>(swl, swh, g4, N, wx0, wy0, cx[0], cy[0], dxl[0],
                                                dyl[0], sv[0]);
                    if (cx[1] >= 0)
                        deposit_fix_one<WX, WY>(swl, swh, g4, N, wx0, wy0, cx[1], cy[1], dxl[1],
                                                dyl[1], sv[1]);
                }
            } else if (joint) {
                // the rows of the stencil in a rolled loop (the x weights
                // move down one register per row): a fifth of the code,
                // which keeps the stage's hot path within the instruction
                // cache
                double ax[5], ay[5], bx[5], by[5];
                weights4(dxl[0], ax); weights4(dyl[0], ay);
                weights4(dxl[1], bx); weights4(dyl[1], by);
                int row = lx * WY + ly;
#pragma unroll 1
                for (int a = 0; a < 5; a++) {
                    const double xa = ax[0], xb = bx[0];
#pragma unroll
                    for (int b = 0; b < 5; b++) {
                        const double wa = xa * ay[b], wb = xb * by[b];
#pragma unroll
                        for (int q = 0; q < 4; q++)
                            shared_fix_add(swl, swh, q * WSZ + row + b,
                                           fma(sv[0][q], wa, fma(sv[1][q], wb, FIX_MAGIC)));
                    }
#pragma unroll
                    for (int k = 0; k < 4; k++) { ax[k] = ax[k + 1]; bx[k] = bx[k + 1]; }
                    row += WY;
                }
            }
        }
    } else {
        const int lx = cx[0] - 2 - wx0, ly = cy[0] - 2 - wy0;
        const bool joint = cx[0] >= 0 && cx[0] == cx[1] && cy[0] == cy[1] &&
                           lx >= 0 && lx + 5 <= WX && ly >= 0 && ly + 5 <= WY;
        double mj = 0;
#pragma unroll
        for (int q = 0; q < 4; q++) mj = fmax(mj, fabs(sv[0][q]) + fabs(sv[1][q]));
        const bool ok = mj * (0.36 * ih * ih) < FIX56_LIMIT;
        if (!__all_sync(0xffffffffu, (joint && ok) || didle)) {
            if (dpair && ok) {
                double ax[6], ay[6], bx[6], by[6], t[5];
                weights4(dxl[0], t); shift6(t, cx[0] - mcx, ax);
                weights4(dyl[0], t); shift6(t, cy[0] - mcy, ay);
                weights4(dxl[1], t); shift6(t, cx[1] - mcx, bx);
                weights4(dyl[1], t); shift6(t, cy[1] - mcy, by);
#pragma unroll
                for (int b = 0; b < 6; b++) { ay[b] *= ih; by[b] *= ih; }
                int row = dx0 * WY + dy0;
#pragma unroll 1
                for (int a = 0; a < 6; a++) {
                    const double xa = ax[0] * ih, xb = bx[0] * ih;
#pragma unroll
                    for (int b = 0; b < 6; b++) {
                        const double wa = xa * ay[b], wb = xb * by[b];
#pragma unroll
                        for (int q = 0; q < 4; q++)
                            fix56_add(swl, sw1, sw2, q * WSZ + row + b, fma(sv[0][q], wa, sv[1][q] * wb));
                    }
#pragma unroll
                    for (int k = 0; k < 5; k++) { ax[k] = ax[k + 1]; bx[k] = bx[k + 1]; }
                    row += WY;
                }
            } else {
#pragma unroll
                for (int p = 0; p < 2; p++)
                    if (cx[p] >= 0)
                        deposit_fix56_one<WX, WY>(swl, sw1, sw2, g4, N, ih, wx0, wy0, cx[p], cy[p],
                                                  dxl[p], dyl[p], sv[p]);
            }
        } else if (joint && ok) {
            // the two contributions summed before the fixed-point atomics;
            // the rows of the stencil in a rolled loop (the x weights move
            // down one register per row): a fifth of the code, which keeps
            // the stage's hot path within the instruction cache
            double ax[5], ay[5], bx[5], by[5];
            weights4(dxl[0], ax); weights4(dyl[0], ay);
            weights4(dxl[1], bx); weights4(dyl[1], by);
#pragma unroll
            for (int b = 0; b < 5; b++) { ay[b] *= ih; by[b] *= ih; }
            int row = lx * WY + ly;
#pragma unroll 1
            for (int a = 0; a < 5; a++) {
                const double xa = ax[0] * ih, xb = bx[0] * ih;
#pragma unroll
                for (int b = 0; b < 5; b++) {
                    const double wa = xa * ay[b], wb = xb * by[b];
#pragma unroll
                    for (int q = 0; q < 4; q++)
                        fix56_add(swl, sw1, sw2, q * WSZ + row + b, fma(sv[0][q], wa, sv[1][q] * wb));
                }
#pragma unroll
                for (int k = 0; k < 4; k++) { ax[k] = ax[k + 1]; bx[k] = bx[k + 1]; }
                row += WY;
            }
        }
    }
    __syncthreads();
    for (int t = threadIdx.x; t < WSZ; t += blockDim.x) {
        const int gx = wx0 + t / WY, gy = wy0 + t % WY;
        if (gx < 0 || gx >= N || gy < 0 || gy >= N) continue;
        const int64_t c = (int64_t)gx * N + gy;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            if constexpr (MIXED) {
                const long long v = ((long long)swh[q * WSZ + t] << 20) + (long long)swl[q * WSZ + t];
                if (v) atomicAdd(g4[q] + c, (fix_t)v);
            } else {
                const int i = q * WSZ + t;
                if (swl[i] | sw1[i] | (unsigned)sw2[i])
                    atomicAdd(g4[q] + c, fix56_value(swl[i], sw1[i], sw2[i]));
            }
        }
    }
}

template <typename FT, int WX, int WY>
static size_t move_deposit_pair_smem()
{
    // deposit window: two 32-bit words per sum (mixed), three (FP64)
    return (size_t)WX * WY * (FieldWin<FT>::bytes_per_cell + 4 * 4 * (sizeof(FT) == 4 ? 2 : 3));
}

template <typename FT, int WX, int WY, bool FIRST>
static int launch_move_deposit_pair(const lcb_move_deposit_args *a, dim3 grid,
                                    typename StageAcc<FT>::type *const out[4], cudaStream_t st)
{
    const size_t sm = move_deposit_pair_smem<FT, WX, WY>();
    static std::atomic<unsigned long long> attr{0};
    {
        const cudaError_t e = ensure_smem(k_move_deposit_pair<FT, WX, WY, FIRST>, sm, attr);
        if (e != cudaSuccess) return cuda_check(e, "move_deposit smem attribute");
    }
    const lcb_plasma_particles &p = a->prev, &f = a->full;
    const cudaError_t e = launch_after(
        k_move_deposit_pair<FT, WX, WY, FIRST>, grid, dim3(DEP_THREADS), sm, st,
        a->n_per_sort, a->particles_side, a->grid_steps, a->h, a->xi_step, a->boundary,
        a->fields[0], a->fields[1], a->fields[2], a->fields[3], a->fields[4], a->fields[5],
        p.x_init, p.y_init, p.x_offt, p.y_offt, p.px, p.py, p.pz, p.q, p.m,
        f.q, f.x_offt, f.y_offt, f.px, f.py, f.pz, out[0], out[1], out[2], out[3], a->err);
    if (e != cudaSuccess) return cuda_check(e, "move_deposit launch");
    return LCB_OK;
}

// Window: the tile's cells (8 x 16 with two or more particles per cell,
// 16 x 32 with one) + 2 stencil + 4 slack on each side.
template <typename FT>
static int dispatch_move_deposit_pair(const lcb_move_deposit_args *a,
                                      typename StageAcc<FT>::type *const out[4], cudaStream_t st)
{
    const dim3 grid((a->particles_side + DEP_TJ - 1) / DEP_TJ,
                    (a->particles_side + 1 + DEP_TI - 1) / DEP_TI,   // spare tile row
                    a->n_sorts);
    if (a->lattice_fineness >= 2)
        return a->first ? launch_move_deposit_pair<FT, 20, 28, true>(a, grid, out, st)
                        : launch_move_deposit_pair<FT, 20, 28, false>(a, grid, out, st);
    return a->first ? launch_move_deposit_pair<FT, DEP_WX, DEP_WY, true>(a, grid, out, st)
                    : launch_move_deposit_pair<FT, DEP_WX, DEP_WY, false>(a, grid, out, st);
}

// Fixed-point sums (4 quantities x 2 columns x N*N) to the FP64 outputs;
// columns past n_sorts get the background ions (ro) or zero.  A thread
// takes one node of both columns.
__global__ void k_fix_finish(int64_t plane, int n_sorts, const fix_t *__restrict__ w,
                             const double *__restrict__ ro_initial, double *ro, double *jx,
                             double *jy, double *jz)
{
    pdl_wait();
    double *outs[4] = {ro, jx, jy, jz};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < plane;
         t += (int64_t)gridDim.x * blockDim.x) {
        double v[8];
#pragma unroll
        for (int qd = 0; qd < 4; qd++) {
            v[2 * qd] = (double)(long long)w[qd * 2 * plane + t] * FIX_INV;
            v[2 * qd + 1] = n_sorts > 1 ? (double)(long long)w[qd * 2 * plane + plane + t] * FIX_INV
                          : ((qd == 0 && ro_initial) ? ro_initial[t] : 0.0);
        }
#pragma unroll
        for (int qd = 0; qd < 4; qd++) {
            outs[qd][t] = v[2 * qd];
            outs[qd][plane + t] = v[2 * qd + 1];
        }
    }
}

// Zero four regions of n 8-byte words each (one kernel in the stream's chain
// of programmatic launches, where a memset would break it).
__global__ void __launch_bounds__(256) k_zero4(uint64_t *r0, uint64_t *r1, uint64_t *r2, uint64_t *r3,
                                               int64_t n)
{
    pdl_wait();
    pdl_trigger();
    uint64_t *r[4] = {r0, r1, r2, r3};
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n;
         t += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int q = 0; q < 4; q++) r[q][t] = 0ull;
    }
}

static int grid_for(int64_t n, int threads);

static int zero4(void *r0, void *r1, void *r2, void *r3, int64_t n, cudaStream_t st)
{
    const cudaError_t e = launch_after(k_zero4, dim3(grid_for(n, 256)), dim3(256), 0, st,
                                       static_cast<uint64_t *>(r0), static_cast<uint64_t *>(r1),
                                       static_cast<uint64_t *>(r2), static_cast<uint64_t *>(r3), n);
    if (e != cudaSuccess) return cuda_check(e, "zero launch");
    count_launch();
    return LCB_OK;
}

// Zero the columns of the fixed-point sums that the deposit adds to (the
// first column of each quantity, both with two sorts).
static int clear_fixed(fix_t *w, size_t plane, int n_sorts, cudaStream_t st)
{
    const int64_t n = (int64_t)(n_sorts > 1 ? 2 : 1) * plane;
    return zero4(w, w + 2 * plane, w + 4 * plane, w + 6 * plane, n, st);
}

static int grid_for(int64_t n, int threads)
{
    int64_t blocks = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count() * 16;
    if (blocks > cap) blocks = cap;
    return (int)(blocks < 1 ? 1 : blocks);
}

// Mixed-precision deposit: fixed-point sums in the workspace, then one pass
// to the FP64 outputs (background column included).
static int deposit_fixed(int64_t n_per_sort, int n_sorts, int N, double h, int particles_side,
                         const double *x_init, const double *y_init, const double *x_offt,
                         const double *y_offt, const double *px, const double *py,
                         const double *pz, const double *q, const double *m,
                         const double *ro_initial, double *ro, double *jx, double *jy,
                         double *jz, void *workspace, size_t workspace_bytes, int *err,
                         cudaStream_t st)
{
    const size_t plane = (size_t)N * N;
    LCB_REQUIRE(workspace && workspace_bytes >= (size_t)8 * plane * sizeof(fix_t),
                "deposit workspace too small");
    fix_t *w = static_cast<fix_t *>(workspace);
    int rc = clear_fixed(w, plane, n_sorts, st);
    if (rc) return rc;
    cudaError_t e;
    if (n_per_sort > 0) {
        const dim3 grid((particles_side + DEP_TJ - 1) / DEP_TJ,
                        (particles_side + 1 + DEP_TI - 1) / DEP_TI, n_sorts);   // spare tile row
        const size_t sm = deposit_smem_bytes<fix_t>();
        static std::atomic<unsigned long long> attr{0};
        e = ensure_smem(k_deposit_tiled<fix_t>, sm, attr);
        if (e != cudaSuccess) return cuda_check(e, "deposit smem attribute");
        k_deposit_tiled<fix_t><<<grid, DEP_THREADS, sm, st>>>(
            n_per_sort, particles_side, N, h, x_init, y_init, x_offt, y_offt, px, py, pz, q, m,
            w, w + 2 * plane, w + 4 * plane, w + 6 * plane, err);
        LCB_LAUNCH_CHECK("k_deposit_tiled<fixed>");
    }
    e = launch_after(k_fix_finish, dim3(grid_for(plane, 256)), dim3(256), 0, st, (int64_t)plane,
                     n_sorts, (const fix_t *)w, ro_initial, ro, jx, jy, jz);
    if (e != cudaSuccess) return cuda_check(e, "fix finish launch");
    count_launch();
    return LCB_OK;
}

}  // namespace lcb

using namespace lcb;

extern "C" int lcb_plasma_move_wo_fields(
    int64_t n, double xi_step, const double *m, const double *x_offt_prev,
    const double *y_offt_prev, const double *px_prev, const double *py_prev,
    const double *pz_prev, const double *q_prev, double *x_offt_full,
    double *y_offt_full, double *px_full, double *py_full, double *pz_full,
    double *q_full, void *stream)
{
    LCB_REQUIRE(n >= 0, "n < 0");
    if (n == 0) return LCB_OK;
    k_move_wo_fields<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(
        n, xi_step, m, x_offt_prev, y_offt_prev, px_prev, py_prev, pz_prev,
        q_prev, x_offt_full, y_offt_full, px_full, py_full, pz_full, q_full);
    LCB_LAUNCH_CHECK("k_move_wo_fields");
    return LCB_OK;
}

extern "C" int lcb_plasma_move_smart(
    int64_t n, double xi_step, double boundary, double h, int grid_steps,
    const double *Ex, const double *Ey, const double *Ez, const double *Bx,
    const double *By, const double *Bz, const double *x_init,
    const double *y_init, const double *x_offt_prev, const double *y_offt_prev,
    const double *px_prev, const double *py_prev, const double *pz_prev,
    const double *m, double *q_full, double *x_offt_full, double *y_offt_full,
    double *px_full, double *py_full, double *pz_full, int *err, void *stream)
{
    LCB_REQUIRE(n >= 0 && grid_steps >= 5, "bad sizes n=%lld N=%d", (long long)n, grid_steps);
    if (n == 0) return LCB_OK;
    k_move_smart<<<grid_for(n, 256), 256, 0, as_stream(stream)>>>(
        n, xi_step, boundary, h, grid_steps, Ex, Ey, Ez, Bx, By, Bz, x_init,
        y_init, x_offt_prev, y_offt_prev, px_prev, py_prev, pz_prev, m, q_full,
        x_offt_full, y_offt_full, px_full, py_full, pz_full, err);
    LCB_LAUNCH_CHECK("k_move_smart");
    return LCB_OK;
}

extern "C" size_t lcb_plasma_deposit_workspace_bytes(int grid_steps, int precision)
{
    if (precision == LCB_PREC_MIXED)
        return (size_t)8 * grid_steps * grid_steps * sizeof(fix_t);
    return 0;
}

extern "C" int lcb_plasma_deposit(
    int64_t n_per_sort, int n_sorts, int grid_steps, double h, int particles_side,
    int precision, const double *x_init, const double *y_init,
    const double *x_offt, const double *y_offt, const double *px,
    const double *py, const double *pz, const double *q, const double *m,
    const double *ro_initial, double *ro, double *jx, double *jy, double *jz,
    void *workspace, size_t workspace_bytes, int *err, void *stream)
{
    const int N = grid_steps;
    LCB_REQUIRE(n_sorts >= 1 && n_sorts <= 2, "n_sorts must be 1 or 2");
    LCB_REQUIRE((int64_t)particles_side * particles_side == n_per_sort,
                "n_per_sort (%lld) must be particles_side^2 (%d^2)",
                (long long)n_per_sort, particles_side);
    LCB_REQUIRE(N >= 5, "grid_steps < 5");
    LCB_REQUIRE(precision == LCB_PREC_FP64 || precision == LCB_PREC_MIXED, "bad precision");
    cudaStream_t st = as_stream(stream);
    const size_t plane = (size_t)N * N;
    const size_t bytes = 2 * plane * sizeof(double);
    if (precision == LCB_PREC_MIXED)
        return deposit_fixed(n_per_sort, n_sorts, N, h, particles_side, x_init, y_init, x_offt,
                             y_offt, px, py, pz, q, m, ro_initial, ro, jx, jy, jz, workspace,
                             workspace_bytes, err, st);
    for (double *p : {ro, jx, jy, jz}) {
        cudaError_t e = cudaMemsetAsync(p, 0, bytes, st);
        if (e != cudaSuccess) return cuda_check(e, "memset currents");
    }
    if (n_per_sort > 0) {
        dim3 grid((particles_side + DEP_TJ - 1) / DEP_TJ,
                  (particles_side + 1 + DEP_TI - 1) / DEP_TI, n_sorts);   // spare tile row
        {
            const size_t sm = deposit_smem_bytes<double>();
            static std::atomic<unsigned long long> attr{0};
            const cudaError_t e = ensure_smem(k_deposit_tiled<double>, sm, attr);
            if (e != cudaSuccess) return cuda_check(e, "deposit smem attribute");
            k_deposit_tiled<double><<<grid, DEP_THREADS, sm, st>>>(
                n_per_sort, particles_side, N, h, x_init, y_init, x_offt, y_offt,
                px, py, pz, q, m, ro, jx, jy, jz, err);
            LCB_LAUNCH_CHECK("k_deposit_tiled<double>");
        }
    }
    if (ro_initial) {
        cudaError_t e = cudaMemcpyAsync(ro + plane, ro_initial, plane * sizeof(double),
                                        cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_check(e, "copy ro_initial");
    }
    return LCB_OK;
}

extern "C" int lcb_plasma_move_deposit(const lcb_move_deposit_args *a, void *stream)
{
    LCB_REQUIRE(a, "args is NULL");
    const int N = a->grid_steps;
    LCB_REQUIRE(a->n_sorts >= 1 && a->n_sorts <= 2, "n_sorts must be 1 or 2");
    LCB_REQUIRE((int64_t)a->particles_side * a->particles_side == a->n_per_sort,
                "n_per_sort (%lld) must be particles_side^2 (%d^2)",
                (long long)a->n_per_sort, a->particles_side);
    LCB_REQUIRE(N >= 5, "grid_steps < 5");
    LCB_REQUIRE(a->precision == LCB_PREC_FP64 || a->precision == LCB_PREC_MIXED, "bad precision");
    for (int f = 0; f < 6; f++) LCB_REQUIRE(a->fields[f], "field plane %d is NULL", f);
    cudaStream_t st = as_stream(stream);
    const size_t plane = (size_t)N * N;
    if (a->precision == LCB_PREC_MIXED) {
        LCB_REQUIRE(a->workspace && a->workspace_bytes >= lcb_plasma_deposit_workspace_bytes(N, a->precision),
                    "deposit workspace too small");
        fix_t *w = static_cast<fix_t *>(a->workspace);
        const int rc0 = clear_fixed(w, plane, a->n_sorts, st);
        if (rc0) return rc0;
        if (a->n_per_sort > 0) {
            fix_t *const out[4] = {w, w + 2 * plane, w + 4 * plane, w + 6 * plane};
            const int rc = dispatch_move_deposit_pair<float>(a, out, st);
            if (rc) return rc;
            LCB_LAUNCH_CHECK("k_move_deposit_pair<float>");
        }
        const cudaError_t e = launch_after(k_fix_finish, dim3(grid_for(plane, 256)), dim3(256), 0, st,
                                           (int64_t)plane, a->n_sorts, (const fix_t *)w,
                                           a->ro_initial, a->ro, a->jx, a->jy, a->jz);
        if (e != cudaSuccess) return cuda_check(e, "fix finish launch");
        count_launch();
        return LCB_OK;
    }
    {
        const int rc0 = zero4(a->ro, a->jx, a->jy, a->jz, 2 * (int64_t)plane, st);
        if (rc0) return rc0;
    }
    if (a->n_per_sort > 0) {
        double *const out[4] = {a->ro, a->jx, a->jy, a->jz};
        const int rc = dispatch_move_deposit_pair<double>(a, out, st);
        if (rc) return rc;
        LCB_LAUNCH_CHECK("k_move_deposit_pair<double>");
    }
    if (a->ro_initial) {
        cudaError_t e = cudaMemcpyAsync(a->ro + plane, a->ro_initial, plane * sizeof(double),
                                        cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return cuda_check(e, "copy ro_initial");
    }
    return LCB_OK;
}
