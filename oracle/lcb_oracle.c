/*
 * CPU oracle for the quasistatic 3D xi step -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C, the per-particle loops of the reference
 * lcodePy 3D path so that the CUDA product can be checked against it.  It is
 * never linked into the product library; only tests/, the smoke check and
 * bench.py's CPU-baseline arm load it (through oracle/oracle.py).
 *
 * Each function cites the reference routine whose arithmetic it follows
 * (paths are relative to the lcodePy project root).  Arithmetic is FP64 and
 * follows the reference's operation order; the build uses -ffp-contract=off
 * so that no fused multiply-adds change the rounding.
 *
 * Loops that are prange-parallel in the reference (the plasma pushers) use
 * OpenMP here too; the depositions are serial, exactly as in the reference.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* 4th-order spline weight for stencil offset `place` in -2..2.
 * lcode/plasma3d/weights.py:13-31 (CPU) and :127-148 (GPU string). */
static inline double w4(double x, int place)
{
    switch (place) {
    case -2: { double a = 0.5 - x; return a * a * a * a / 24.0; }
    case -1: return 19.0 / 96.0 - 11.0 / 24.0 * x + x * x / 4.0
                    + x * x * x / 6.0 - x * x * x * x / 6.0;
    case 0:  return 115.0 / 192.0 - 5.0 / 8.0 * x * x + x * x * x * x / 4.0;
    case 1:  return 19.0 / 96.0 + 11.0 / 24.0 * x + x * x / 4.0
                    - x * x * x / 6.0 - x * x * x * x / 6.0;
    case 2:  { double a = 0.5 + x; return a * a * a * a / 24.0; }
    default: return 0.0;
    }
}

/* Linear weight in xi.  lcode/beam3d/weights.py:9-14 / :251-260. */
static inline double w1(double x, int place)
{
    return place == 0 ? x : 1.0 - x;
}

/* Error counter for stencil points outside the N*N grid (the reference does
 * not check; the oracle skips such points and counts them). */
static int64_t g_oob = 0;
int64_t orc_oob_count(void) { return g_oob; }
void orc_oob_reset(void) { g_oob = 0; }

/* Free-streaming estimate x_offt += px/(gamma m - pz) dxi.
 * lcode/plasma3d/move.py:151-165 (CPU), :292-313 (GPU). */
void orc_move_wo_fields(int64_t n, double xi_step, const double *m,
                        double *x_offt, double *y_offt, const double *px,
                        const double *py, const double *pz)
{
    int64_t k;
#pragma omp parallel for schedule(static)
    for (k = 0; k < n; k++) {
        if (m[k] == 0) continue;
        double gm = sqrt(m[k] * m[k] + pz[k] * pz[k] + px[k] * px[k] + py[k] * py[k]);
        x_offt[k] += px[k] / (gm - pz[k]) * xi_step;
        y_offt[k] += py[k] / (gm - pz[k]) * xi_step;
    }
}

/* Fused midpoint gather + two-pass momentum update + advance + reflection +
 * absorption.  Follows the GPU kernel lcode/plasma3d/move.py:169-289; the CPU
 * twin :52-148 computes the same values in the same order. */
void orc_move_smart(int64_t n, double xi_step, double boundary, double h,
                    int grid_steps,
                    const double *Ex_f, const double *Ey_f, const double *Ez_f,
                    const double *Bx_f, const double *By_f, const double *Bz_f,
                    const double *x_init, const double *y_init,
                    const double *x_offt_prev, const double *y_offt_prev,
                    const double *px_prev, const double *py_prev,
                    const double *pz_prev, const double *m, double *q,
                    double *x_offt_full, double *y_offt_full, double *px_full,
                    double *py_full, double *pz_full)
{
    const int N = grid_steps;
    const int64_t NN = (int64_t)N * N;
    int64_t oob = 0;
    int64_t k;
#pragma omp parallel for schedule(static) reduction(+:oob)
    for (k = 0; k < n; k++) {
        if (q[k] == 0) continue;
        double px = px_prev[k], py = py_prev[k], pz = pz_prev[k];
        double xh = x_init[k] + (x_offt_prev[k] + x_offt_full[k]) / 2;
        double yh = y_init[k] + (y_offt_prev[k] + y_offt_full[k]) / 2;
        if (xh > boundary)  { xh =  2 * boundary - xh; px = py = pz = 0; }
        if (xh < -boundary) { xh = -2 * boundary - xh; px = py = pz = 0; }
        if (yh > boundary)  { yh =  2 * boundary - yh; px = py = pz = 0; }
        if (yh < -boundary) { yh = -2 * boundary - yh; px = py = pz = 0; }

        double x_h = xh / h + 0.5, y_h = yh / h + 0.5;
        double x_loc = x_h - floor(x_h) - 0.5, y_loc = y_h - floor(y_h) - 0.5;
        int ix = (int)(floor(x_h) + N / 2), iy = (int)(floor(y_h) + N / 2);

        double Ex = 0, Ey = 0, Ez = 0, Bx = 0, By = 0, Bz = 0;
        for (int kx = -2; kx <= 2; kx++) {
            double wx = w4(x_loc, kx);
            for (int ky = -2; ky <= 2; ky++) {
                double w = wx * w4(y_loc, ky);
                int gx = ix + kx, gy = iy + ky;
                if (gx < 0 || gx >= N || gy < 0 || gy >= N) { oob++; continue; }
                int64_t idx = gy + (int64_t)N * gx;
                (void)NN;
                Ex += Ex_f[idx] * w; Bx += Bx_f[idx] * w;
                Ey += Ey_f[idx] * w; By += By_f[idx] * w;
                Ez += Ez_f[idx] * w; Bz += Bz_f[idx] * w;
            }
        }

        const double opx = px_prev[k], opy = py_prev[k], opz = pz_prev[k];
        double x_offt = x_offt_prev[k], y_offt = y_offt_prev[k];
        const double mk = m[k], qk = q[k];

        double gm = sqrt(mk * mk + px * px + py * py + pz * pz);
        double vx = px / gm, vy = py / gm, vz = pz / gm;
        double f = qk * xi_step / (1 - pz / gm);
        double dpx = f * (Ex + vy * Bz - vz * By);
        double dpy = f * (Ey - vx * Bz + vz * Bx);
        double dpz = f * (Ez + vx * By - vy * Bx);
        px = opx + dpx / 2; py = opy + dpy / 2; pz = opz + dpz / 2;

        gm = sqrt(mk * mk + px * px + py * py + pz * pz);
        vx = px / gm; vy = py / gm; vz = pz / gm;
        f = qk * xi_step / (1 - pz / gm);
        dpx = f * (Ex + vy * Bz - vz * By);
        dpy = f * (Ey - vx * Bz + vz * Bx);
        dpz = f * (Ez + vx * By - vy * Bx);
        px = opx + dpx / 2; py = opy + dpy / 2; pz = opz + dpz / 2;

        gm = sqrt(mk * mk + px * px + py * py + pz * pz);
        x_offt += px / (gm - pz) * xi_step;
        y_offt += py / (gm - pz) * xi_step;
        px = opx + dpx; py = opy + dpy; pz = opz + dpz;

        double x = x_init[k] + x_offt, y = y_init[k] + y_offt;
        if (x > boundary)  { x =  2 * boundary - x; x_offt = x - x_init[k]; px = py = pz = 0; }
        if (x < -boundary) { x = -2 * boundary - x; x_offt = x - x_init[k]; px = py = pz = 0; }
        if (y > boundary)  { y =  2 * boundary - y; y_offt = y - y_init[k]; px = py = pz = 0; }
        if (y < -boundary) { y = -2 * boundary - y; y_offt = y - y_init[k]; px = py = pz = 0; }
        if (x >= boundary || x <= -boundary || y >= boundary || y <= -boundary) {
            x_offt = y_offt = 0; px = py = pz = 0; q[k] = 0;
        }
        x_offt_full[k] = x_offt; y_offt_full[k] = y_offt;
        px_full[k] = px; py_full[k] = py; pz_full[k] = pz;
    }
    g_oob += oob;
}

/* 25-point deposition of rho, jx, jy, jz, serial in particle order.
 * lcode/plasma3d/weights.py:35-67 (CPU), :151-190 (GPU); x_h, y_h computed
 * as in :249-285. */
void orc_deposit_plasma(int64_t n, int grid_steps, double h,
                        const double *x_init, const double *y_init,
                        const double *x_offt, const double *y_offt,
                        const double *px, const double *py, const double *pz,
                        const double *q, const double *m, double *ro,
                        double *jx, double *jy, double *jz)
{
    const int N = grid_steps;
    for (int64_t k = 0; k < n; k++) {
        if (q[k] == 0) continue;
        double x_h = (x_init[k] + x_offt[k]) / h + 0.5;
        double y_h = (y_init[k] + y_offt[k]) / h + 0.5;
        double gm = sqrt(m[k] * m[k] + px[k] * px[k] + py[k] * py[k] + pz[k] * pz[k]);
        double dro = q[k] / (1 - pz[k] / gm);
        double djx = px[k] * (dro / gm);
        double djy = py[k] * (dro / gm);
        double djz = pz[k] * (dro / gm);
        double x_loc = x_h - floor(x_h) - 0.5, y_loc = y_h - floor(y_h) - 0.5;
        int ix = (int)(floor(x_h) + N / 2), iy = (int)(floor(y_h) + N / 2);
        for (int kx = -2; kx <= 2; kx++) {
            double wx = w4(x_loc, kx) / h;
            for (int ky = -2; ky <= 2; ky++) {
                double w = wx * w4(y_loc, ky) / h;
                int gx = ix + kx, gy = iy + ky;
                if (gx < 0 || gx >= N || gy < 0 || gy >= N) { g_oob++; continue; }
                int64_t idx = gy + (int64_t)N * gx;
                ro[idx] += dro * w;
                jx[idx] += djx * w;
                jy[idx] += djy * w;
                jz[idx] += djz * w;
            }
        }
    }
}

/* Beam density deposit: 25-point transverse x linear in xi, into the carried
 * layer (ro0, weight xi_loc) and the next layer (ro1, weight 1 - xi_loc).
 * lcode/beam3d/weights.py:40-65 (CPU), :108-138 (GPU), driver :152-163.
 * Stencil points whose flat index y + N*x leaves [0, N*N) are skipped and
 * counted; flat indices inside the array are used as the reference does. */
void orc_deposit_beam(int64_t n, int grid_steps, double h, double xi_step,
                      int64_t layer_idx, const double *x, const double *y,
                      const double *xi, const double *q_norm, double *ro0,
                      double *ro1)
{
    const int N = grid_steps;
    const int64_t NN = (int64_t)N * N;
    const double xi_layer = -xi_step * (double)layer_idx;
    for (int64_t k = 0; k < n; k++) {
        double xi_loc = (xi_layer - xi[k]) / xi_step;
        double x_h = x[k] / h + 0.5, y_h = y[k] / h + 0.5;
        double x_loc = x_h - floor(x_h) - 0.5, y_loc = y_h - floor(y_h) - 0.5;
        int ix = (int)(floor(x_h) + N / 2), iy = (int)(floor(y_h) + N / 2);
        for (int kx = -2; kx <= 2; kx++) {
            double wx = w4(x_loc, kx);
            for (int ky = -2; ky <= 2; ky++) {
                double w = wx * w4(y_loc, ky);
                double wa = w * w1(xi_loc, 0);
                double wb = w * w1(xi_loc, 1);
                int64_t idx = (int64_t)(iy + ky) + (int64_t)N * (ix + kx);
                if (idx < 0 || idx >= NN) { g_oob++; continue; }
                ro0[idx] += q_norm[k] * wa;
                ro1[idx] += q_norm[k] * wb;
            }
        }
    }
}

/* Substep size: dt = 1, halved while dt > sqrt(sqrt(1/q_m^2 + pz^2)/E_sub).
 * lcode/beam3d/beam_calculator.py:18-25 (CPU), :28-46 (GPU); the caller
 * scales by time-step and sets remaining_steps = (int)(1/dt) as in :111-114. */
void orc_beam_substepping(int64_t n, const double *q_m, const double *pz,
                          double substep_energy, double time_step, double *dt,
                          int64_t *remaining_steps)
{
    for (int64_t k = 0; k < n; k++) {
        double d = 1.0;
        double max_dt = sqrt(sqrt(1 / (q_m[k] * q_m[k]) + pz[k] * pz[k]) / substep_energy);
        while (d > max_dt) d /= 2;
        dt[k] = d * time_step;
        remaining_steps[k] = (int64_t)(1.0 / d);
    }
}

/* Substepped Higuera-Cary beam push inside one xi layer, with fields linearly
 * weighted between the layer's two plasma planes exactly as the GPU kernel
 * lcode/beam3d/move.py:155-273 weights them (w0 = xi_loc on fields_k,
 * w1 = 1 - xi_loc on fields_k1).  Flags: 1 lost, 2 moved, 4 fell. */
void orc_move_beam(int64_t n, double xi_step, double r_max,
                   int64_t beam_layer_idx, double h, int grid_steps,
                   const double *q_m, const double *dt,
                   const double *Exk, const double *Eyk, const double *Ezk,
                   const double *Bxk, const double *Byk, const double *Bzk,
                   const double *Exk1, const double *Eyk1, const double *Ezk1,
                   const double *Bxk1, const double *Byk1, const double *Bzk1,
                   int64_t *remaining_steps, int64_t *id, double *x, double *y,
                   double *xi, double *px, double *py, double *pz,
                   uint8_t *flags)
{
    const int N = grid_steps;
    const int64_t NN = (int64_t)N * N;
    const double xi_k = (double)beam_layer_idx * (-xi_step);
    const double xi_k1 = (double)(beam_layer_idx + 1) * (-xi_step);
    int64_t oob = 0;
    int64_t i;
#pragma omp parallel for schedule(dynamic, 64) reduction(+:oob)
    for (i = 0; i < n; i++) {
        int lost = 0, fell = 0;
        const double q = copysign(1.0, q_m[i]);
        const double im = 1.0 / q_m[i];
        while (remaining_steps[i] > 0) {
            double gm = sqrt(im * im + px[i] * px[i] + py[i] * py[i] + pz[i] * pz[i]);
            double xh = x[i] + dt[i] / 2.0 * (px[i] / gm);
            double yh = y[i] + dt[i] / 2.0 * (py[i] / gm);
            double xih = xi[i] + dt[i] / 2.0 * (pz[i] / gm - 1);
            if (xih < xi_k1) { fell = 1; break; }
            if (xh * xh + yh * yh >= r_max * r_max) {
                x[i] = xh; y[i] = yh; xi[i] = xih;
                id[i] *= -1; lost = 1; remaining_steps[i] = 0; break;
            }
            double x_h = xh / h + 0.5, y_h = yh / h + 0.5;
            double x_loc = x_h - floor(x_h) - 0.5, y_loc = y_h - floor(y_h) - 0.5;
            double xi_loc = (xih - xi_k) / xi_step;
            int ix = (int)(floor(x_h) + N / 2), iy = (int)(floor(y_h) + N / 2);
            double Ex = 0, Ey = 0, Ez = 0, Bx = 0, By = 0, Bz = 0;
            for (int kx = -2; kx <= 2; kx++) {
                double wx = w4(x_loc, kx);
                for (int ky = -2; ky <= 2; ky++) {
                    double w = wx * w4(y_loc, ky);
                    double wa = w * w1(xi_loc, 0);
                    double wb = w * w1(xi_loc, 1);
                    int64_t idx = (int64_t)(iy + ky) + (int64_t)N * (ix + kx);
                    if (idx < 0 || idx >= NN) { oob++; continue; }
                    Ex += Exk[idx] * wa + Exk1[idx] * wb;
                    Bx += Bxk[idx] * wa + Bxk1[idx] * wb;
                    Ey += Eyk[idx] * wa + Eyk1[idx] * wb;
                    By += Byk[idx] * wa + Byk1[idx] * wb;
                    Ez += Ezk[idx] * wa + Ezk1[idx] * wb;
                    Bz += Bzk[idx] * wa + Bzk1[idx] * wb;
                }
            }
            const double hd = q * dt[i] / 2.0;
            double pxm = px[i] + hd * Ex, bx = hd * Bx;
            double pym = py[i] + hd * Ey, by = hd * By;
            double pzm = pz[i] + hd * Ez, bz = hd * Bz;
            gm = sqrt(im * im + pxm * pxm + pym * pym + pzm * pzm);
            double bsq = bx * bx + by * by + bz * bz;
            double bp = bx * pxm + by * pym + bz * pzm;
            double g2 = gm * gm - bsq;
            gm = sqrt((g2 + sqrt(g2 * g2 + 4 * bsq + 4 * bp * bp)) / 2.0);
            double tx = bx / gm, ty = by / gm, tz = bz / gm;
            double tp = 1.0 + tx * tx + ty * ty + tz * tz;
            double tm = 1.0 - tx * tx - ty * ty - tz * tz;
            double sx = 2.0 * tx / tp, sy = 2.0 * ty / tp, sz = 2.0 * tz / tp;
            double sp = sx * pxm + sy * pym + sz * pzm;
            px[i] = tx * sp + pxm * tm / tp + pym * sz - pzm * sy + hd * Ex;
            py[i] = ty * sp + pym * tm / tp + pzm * sx - pxm * sz + hd * Ey;
            pz[i] = tz * sp + pzm * tm / tp + pxm * sy - pym * sx + hd * Ez;
            gm = sqrt(im * im + px[i] * px[i] + py[i] * py[i] + pz[i] * pz[i]);
            x[i] = xh + dt[i] / 2.0 * (px[i] / gm);
            y[i] = yh + dt[i] / 2.0 * (py[i] / gm);
            xi[i] = xih + dt[i] / 2.0 * (pz[i] / gm - 1);
            if (x[i] * x[i] + y[i] * y[i] >= r_max * r_max) {
                id[i] *= -1; lost = 1; remaining_steps[i] = 0; break;
            }
            remaining_steps[i] -= 1;
        }
        if (remaining_steps[i] == 0 && xi[i] < xi_k1) fell = 1;
        uint8_t fl = 0;
        if (lost) fl |= 1;
        if (fell) fl |= 4;
        if (!fell && !lost) fl |= 2;
        flags[i] = fl;
    }
    g_oob += oob;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
