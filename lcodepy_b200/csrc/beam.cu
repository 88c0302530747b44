// Beam kernels: density deposit of a layer, substep sizes, and the substepped
// Higuera-Cary push of a layer between two plasma planes.  FP64.
#include "common.cuh"

namespace lcb {

// Beam density deposit (lcode/beam3d/weights.py:108-138, driver :152-163):
// q * w4(x) w4(y) * xi_loc into ro0 and * (1 - xi_loc) into ro1.  Stencil
// points are addressed by the flat index (iy+ky) + N (ix+kx) as in the
// reference; points whose flat index leaves [0, N*N) are skipped and flagged.
__global__ void __launch_bounds__(128)
k_beam_deposit(int64_t n, int N, double h, double xi_step, double xi_layer,
               const double *__restrict__ x, const double *__restrict__ y,
               const double *__restrict__ xi, const double *__restrict__ q,
               double *ro0, double *ro1, int *err)
{
    const int half_n = N / 2;
    const int64_t NN = (int64_t)N * N;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const double xi_loc = (xi_layer - xi[k]) / xi_step;
        double xl, yl;
        const int ix = cell_of(x[k] / h + 0.5, half_n, xl);
        const int iy = cell_of(y[k] / h + 0.5, half_n, yl);
        double wx[5], wy[5];
        weights4(xl, wx);
        weights4(yl, wy);
        const double qk = q[k];
        bool bad = false;
#pragma unroll
        for (int a = 0; a < 5; a++) {
#pragma unroll
            for (int b = 0; b < 5; b++) {
                const double w = wx[a] * wy[b];
                const double w0 = w * xi_loc, w1 = w * (1 - xi_loc);
                const int64_t idx = (int64_t)(iy + b - 2) + (int64_t)N * (ix + a - 2);
                if (idx < 0 || idx >= NN) { bad = true; continue; }
                atomicAdd(ro0 + idx, qk * w0);
                atomicAdd(ro1 + idx, qk * w1);
            }
        }
        if (bad && err) atomicOr(err, LCB_DEVERR_BEAM_STENCIL);
    }
}

// Substep size (lcode/beam3d/beam_calculator.py:28-46) and the driver's
// scaling (:111-114).
__global__ void k_beam_substepping(int64_t n, const double *__restrict__ q_m,
                                   const double *__restrict__ pz, double e_sub,
                                   double time_step, double *dt, int64_t *rem)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n;
         k += (int64_t)gridDim.x * blockDim.x) {
        const double qm = q_m[k], p = pz[k];
        const double max_dt = sqrt(sqrt(1 / (qm * qm) + p * p) / e_sub);
        double d = 1.0;
        // The reference halves without limit; here the substep stops at
        // 2^-20 (a million substeps) so a degenerate q_m cannot stall the
        // push kernel.  Physical beams stop after a few halvings.
        while (d > max_dt && d > 0x1p-20) d /= 2;
        dt[k] = d * time_step;
        rem[k] = (int64_t)(1. / d);
    }
}

struct FieldPair {
    const double *k[6], *k1[6];  // Ex Ey Ez Bx By Bz at plane k and k+1
};

// Substepped push (lcode/beam3d/move.py:155-273).  Fields are weighted with
// w0 = xi_loc on plane k and w1 = 1 - xi_loc on plane k+1, as the reference
// GPU kernel weights them.
__global__ void __launch_bounds__(128)
k_beam_move(int64_t n, double xi_step, double r_max, double xi_k, double xi_k1,
            double h, int N, const double *__restrict__ q_m,
            const double *__restrict__ dt_a, FieldPair F, int64_t *rem,
            int64_t *id, double *xa, double *ya, double *xia, double *pxa,
            double *pya, double *pza, uint8_t *flags, int *err)
{
    const int half_n = N / 2;
    const int64_t NN = (int64_t)N * N;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double qm = q_m[i], dt = dt_a[i];
        const double q = copysign(1.0, qm);
        const double im = 1. / qm;
        double x = xa[i], y = ya[i], xi = xia[i], px = pxa[i], py = pya[i], pz = pza[i];
        int64_t r = rem[i];
        bool lost = false, fell = false, bad = false;
        if (r > (int64_t(1) << 20)) {  // bounded work per particle
            r = int64_t(1) << 20;
            if (err) atomicOr(err, LCB_DEVERR_CAPACITY);
        }
        while (r > 0) {
            double gm = sqrt(im * im + px * px + py * py + pz * pz);
            const double xh = x + dt / 2. * (px / gm);
            const double yh = y + dt / 2. * (py / gm);
            const double xih = xi + dt / 2. * (pz / gm - 1);
            if (xih < xi_k1) { fell = true; break; }
            if (xh * xh + yh * yh >= r_max * r_max) {
                x = xh; y = yh; xi = xih;
                lost = true; r = 0;
                break;
            }
            double xl, yl;
            const int ix = cell_of(xh / h + 0.5, half_n, xl);
            const int iy = cell_of(yh / h + 0.5, half_n, yl);
            const double xi_loc = (xih - xi_k) / xi_step;
            double wx[5], wy[5];
            weights4(xl, wx);
            weights4(yl, wy);
            double Ex = 0, Ey = 0, Ez = 0, Bx = 0, By = 0, Bz = 0;
#pragma unroll
            for (int a = 0; a < 5; a++) {
#pragma unroll
                for (int b = 0; b < 5; b++) {
                    const double w = wx[a] * wy[b];
                    const double w0 = w * xi_loc, w1 = w * (1 - xi_loc);
                    const int64_t idx = (int64_t)(iy + b - 2) + (int64_t)N * (ix + a - 2);
                    if (idx < 0 || idx >= NN) { bad = true; continue; }
                    Ex += __ldg(F.k[0] + idx) * w0 + __ldg(F.k1[0] + idx) * w1;
                    Bx += __ldg(F.k[3] + idx) * w0 + __ldg(F.k1[3] + idx) * w1;
                    Ey += __ldg(F.k[1] + idx) * w0 + __ldg(F.k1[1] + idx) * w1;
                    By += __ldg(F.k[4] + idx) * w0 + __ldg(F.k1[4] + idx) * w1;
                    Ez += __ldg(F.k[2] + idx) * w0 + __ldg(F.k1[2] + idx) * w1;
                    Bz += __ldg(F.k[5] + idx) * w0 + __ldg(F.k1[5] + idx) * w1;
                }
            }
            const double hd = q * dt / 2.;
            const double pxm = px + hd * Ex, bx = hd * Bx;
            const double pym = py + hd * Ey, by = hd * By;
            const double pzm = pz + hd * Ez, bz = hd * Bz;
            gm = sqrt(im * im + pxm * pxm + pym * pym + pzm * pzm);
            const double bsq = bx * bx + by * by + bz * bz;
            const double bp = bx * pxm + by * pym + bz * pzm;
            const double g2 = gm * gm - bsq;
            gm = sqrt((g2 + sqrt(g2 * g2 + 4 * bsq + 4 * bp * bp)) / 2.);
            const double tx = bx / gm, ty = by / gm, tz = bz / gm;
            const double tp = 1. + tx * tx + ty * ty + tz * tz;
            const double tmn = 1. - tx * tx - ty * ty - tz * tz;
            const double sx = 2. * tx / tp, sy = 2. * ty / tp, sz = 2. * tz / tp;
            const double sp = sx * pxm + sy * pym + sz * pzm;
            px = tx * sp + pxm * tmn / tp + pym * sz - pzm * sy + hd * Ex;
            py = ty * sp + pym * tmn / tp + pzm * sx - pxm * sz + hd * Ey;
            pz = tz * sp + pzm * tmn / tp + pxm * sy - pym * sx + hd * Ez;
            gm = sqrt(im * im + px * px + py * py + pz * pz);
            x = xh + dt / 2. * (px / gm);
            y = yh + dt / 2. * (py / gm);
            xi = xih + dt / 2. * (pz / gm - 1);
            if (x * x + y * y >= r_max * r_max) { lost = true; r = 0; break; }
            r -= 1;
        }
        if (r == 0 && xi < xi_k1) fell = true;
        if (lost) id[i] = -id[i];
        xa[i] = x; ya[i] = y; xia[i] = xi; pxa[i] = px; pya[i] = py; pza[i] = pz;
        rem[i] = r;
        flags[i] = (uint8_t)((lost ? 1 : 0) | (fell ? 4 : 0) | (!fell && !lost ? 2 : 0));
        if (bad && err) atomicOr(err, LCB_DEVERR_BEAM_STENCIL);
    }
}

static int grid_for(int64_t n, int threads)
{
    int64_t blocks = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count() * 16;
    if (blocks > cap) blocks = cap;
    return (int)(blocks < 1 ? 1 : blocks);
}

}  // namespace lcb

using namespace lcb;

extern "C" int lcb_beam_deposit(int64_t n, int grid_steps, double h, double xi_step,
                                int64_t layer_idx, const double *x, const double *y,
                                const double *xi, const double *q_norm, double *ro0,
                                double *ro1, int *err, void *stream)
{
    LCB_REQUIRE(n >= 0 && grid_steps >= 5, "bad sizes");
    if (n == 0) return LCB_OK;
    const double xi_layer = -xi_step * (double)layer_idx;
    k_beam_deposit<<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(
        n, grid_steps, h, xi_step, xi_layer, x, y, xi, q_norm, ro0, ro1, err);
    LCB_LAUNCH_CHECK("k_beam_deposit");
    return LCB_OK;
}

extern "C" int lcb_beam_substepping(int64_t n_fresh, const double *q_m, const double *pz,
                                    double substep_energy, double time_step, double *dt,
                                    int64_t *remaining_steps, void *stream)
{
    LCB_REQUIRE(n_fresh >= 0, "n < 0");
    LCB_REQUIRE(substep_energy > 0, "beam-substepping-energy must be > 0");
    if (n_fresh == 0) return LCB_OK;
    k_beam_substepping<<<grid_for(n_fresh, 128), 128, 0, as_stream(stream)>>>(
        n_fresh, q_m, pz, substep_energy, time_step, dt, remaining_steps);
    LCB_LAUNCH_CHECK("k_beam_substepping");
    return LCB_OK;
}

extern "C" int lcb_beam_move(int64_t n, double xi_step, double r_max,
                             int64_t beam_layer_idx, double h, int grid_steps,
                             const double *q_m, const double *dt,
                             const lcb_fields *fields_k, const lcb_fields *fields_k1,
                             int64_t *remaining_steps, int64_t *id, double *x,
                             double *y, double *xi, double *px, double *py,
                             double *pz, uint8_t *flags, int *err, void *stream)
{
    LCB_REQUIRE(n >= 0 && grid_steps >= 5, "bad sizes");
    LCB_REQUIRE(fields_k && fields_k1, "fields are NULL");
    if (n == 0) return LCB_OK;
    FieldPair F;
    for (int c = 0; c < 6; c++) {
        F.k[c] = fields_k->f[c];
        F.k1[c] = fields_k1->f[c];
        LCB_REQUIRE(F.k[c] && F.k1[c], "field plane %d is NULL", c);
    }
    const double xi_k = (double)beam_layer_idx * (-xi_step);
    const double xi_k1 = (double)(beam_layer_idx + 1) * (-xi_step);
    k_beam_move<<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(
        n, xi_step, r_max, xi_k, xi_k1, h, grid_steps, q_m, dt, F,
        remaining_steps, id, x, y, xi, px, py, pz, flags, err);
    LCB_LAUNCH_CHECK("k_beam_move");
    return LCB_OK;
}
