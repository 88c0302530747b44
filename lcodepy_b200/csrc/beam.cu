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

struct PushParams {
    double xi_step, r_max, xi_k, xi_k1, h;
    int N;
};

// One particle's substepped push (lcode/beam3d/move.py:155-273).  Fields are
// weighted with w0 = xi_loc on plane k and w1 = 1 - xi_loc on plane k+1, as
// the reference GPU kernel weights them.  Updates the state in place and
// returns the flags 1 lost | 2 moved | 4 fell; the id is negated when lost.
__device__ uint8_t push_particle(const PushParams &P, const FieldPair &F, double qm, double dt,
                                 int64_t &r, int64_t &id, double &x, double &y, double &xi,
                                 double &px, double &py, double &pz, int *err)
{
    const int half_n = P.N / 2;
    const int64_t NN = (int64_t)P.N * P.N;
    const double q = copysign(1.0, qm);
    const double im = 1. / qm;
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
        if (xih < P.xi_k1) { fell = true; break; }
        if (xh * xh + yh * yh >= P.r_max * P.r_max) {
            x = xh; y = yh; xi = xih;
            lost = true; r = 0;
            break;
        }
        double xl, yl;
        const int ix = cell_of(xh / P.h + 0.5, half_n, xl);
        const int iy = cell_of(yh / P.h + 0.5, half_n, yl);
        const double xi_loc = (xih - P.xi_k) / P.xi_step;
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
                const int64_t idx = (int64_t)(iy + b - 2) + (int64_t)P.N * (ix + a - 2);
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
        if (x * x + y * y >= P.r_max * P.r_max) { lost = true; r = 0; break; }
        r -= 1;
    }
    if (r == 0 && xi < P.xi_k1) fell = true;
    if (lost) id = -id;
    if (bad && err) atomicOr(err, LCB_DEVERR_BEAM_STENCIL);
    return (uint8_t)((lost ? 1 : 0) | (fell ? 4 : 0) | (!fell && !lost ? 2 : 0));
}

__global__ void __launch_bounds__(128)
k_beam_move(int64_t n, PushParams P, const double *__restrict__ q_m,
            const double *__restrict__ dt_a, FieldPair F, int64_t *rem,
            int64_t *id, double *xa, double *ya, double *xia, double *pxa,
            double *pya, double *pza, uint8_t *flags, int *err)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double x = xa[i], y = ya[i], xi = xia[i], px = pxa[i], py = pya[i], pz = pza[i];
        int64_t r = rem[i], pid = id[i];
        flags[i] = push_particle(P, F, q_m[i], dt_a[i], r, pid, x, y, xi, px, py, pz, err);
        xa[i] = x; ya[i] = y; xia[i] = xi; pxa[i] = px; pya[i] = py; pza[i] = pz;
        rem[i] = r;
        id[i] = pid;
    }
}

// ---------------------------------------------------------------------------
// Device-resident layer step: push the previous layer (the fresh particles
// of the source slice, with their substep sizes, then the particles that
// fell from the push before) into a staging buffer, then compact it in order
// into the drain (moved), the next fell buffer and the lost buffer.  The fell
// and drain counts live on the device, so the xi loop never waits for the
// host.  Orders match the reference's boolean-mask gathers
// (beam_calculator.py:130-134, data.py:151-178).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double substep(double qm, double pz, double e_sub)
{
    const double max_dt = sqrt(sqrt(1 / (qm * qm) + pz * pz) / e_sub);
    double d = 1.0;
    while (d > max_dt && d > 0x1p-20) d /= 2;
    return d;
}

struct StepArgs {
    lcb_beam_soa src, fin, stage;
    int64_t move_begin, n_fresh;
    const int64_t *fell_in_count;
    int64_t stage_capacity;
    uint8_t *flags;
    double e_sub, time_step;
    PushParams P;
    FieldPair F;
    double *clear;          // plane zeroed by the same grid (the next layout's lower plane)
    int64_t clear_n;
    int *err;
};

__device__ __forceinline__ void soa_load(const lcb_beam_soa &s, int64_t i, double *v, int64_t &id,
                                         int64_t &rem)
{
    v[0] = s.xi[i]; v[1] = s.x[i]; v[2] = s.y[i]; v[3] = s.px[i]; v[4] = s.py[i];
    v[5] = s.pz[i]; v[6] = s.q_m[i]; v[7] = s.q_norm[i]; v[8] = s.dt[i];
    id = s.id[i];
    rem = s.remaining_steps[i];
}

__device__ __forceinline__ void soa_store(const lcb_beam_soa &s, int64_t i, const double *v,
                                          int64_t id, int64_t rem)
{
    s.xi[i] = v[0]; s.x[i] = v[1]; s.y[i] = v[2]; s.px[i] = v[3]; s.py[i] = v[4];
    s.pz[i] = v[5]; s.q_m[i] = v[6]; s.q_norm[i] = v[7]; s.dt[i] = v[8];
    s.id[i] = id;
    s.remaining_steps[i] = rem;
}

__global__ void __launch_bounds__(128) k_beam_push_stage(StepArgs a)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < a.clear_n;
         t += (int64_t)gridDim.x * blockDim.x)
        a.clear[t] = 0.0;
    const int64_t total = a.n_fresh + *a.fell_in_count;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        if (t >= a.stage_capacity) {
            if (a.err) atomicOr(a.err, LCB_DEVERR_CAPACITY);
            break;
        }
        double v[9];
        int64_t id, rem;
        if (t < a.n_fresh) {
            soa_load(a.src, a.move_begin + t, v, id, rem);
            const double d = substep(v[6], v[5], a.e_sub);  // beam_calculator.py:109-114
            v[8] = d * a.time_step;
            rem = (int64_t)(1. / d);
        } else {
            soa_load(a.fin, t - a.n_fresh, v, id, rem);
        }
        a.flags[t] = push_particle(a.P, a.F, v[6], v[8], rem, id, v[1], v[2], v[0], v[3],
                                   v[4], v[5], a.err);
        soa_store(a.stage, t, v, id, rem);
    }
}

struct CompactArgs {
    lcb_beam_soa stage, drain, fout, lost;
    const uint8_t *flags;
    int64_t n_fresh;
    const int64_t *fell_in_count;
    int64_t stage_capacity;
    int64_t *drain_count, *fell_out_count, *lost_count;
    int64_t drain_capacity, fell_capacity, lost_capacity;
    int *err;
};

constexpr int CMP_THREADS = 1024;

// Ordered compaction by one CTA: an exclusive scan of three 20-bit counters
// packed in a 64-bit word per chunk of 1024 staged particles.
__global__ void __launch_bounds__(CMP_THREADS) k_beam_compact(CompactArgs a)
{
    __shared__ unsigned long long warp_sums[CMP_THREADS / 32];
    __shared__ long long base[3];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int64_t total = a.n_fresh + *a.fell_in_count;
    if (total > a.stage_capacity) total = a.stage_capacity;
    if (tid == 0) {
        base[0] = *a.drain_count;
        base[1] = 0;
        base[2] = a.lost_count ? *a.lost_count : 0;
    }
    __syncthreads();
    for (int64_t c0 = 0; c0 < total; c0 += CMP_THREADS) {
        const int64_t t = c0 + tid;
        const uint8_t f = t < total ? a.flags[t] : 0;
        const unsigned long long mine = (unsigned long long)((f & 2) ? 1 : 0) |
                                        ((unsigned long long)((f & 4) ? 1 : 0) << 20) |
                                        ((unsigned long long)((f & 1) ? 1 : 0) << 40);
        unsigned long long incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_sums[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const unsigned long long v = warp_sums[lane];
            unsigned long long s = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warp_sums[lane] = s - v;  // exclusive over warps
        }
        __syncthreads();
        const unsigned long long excl = warp_sums[warp] + incl - mine;
        const int64_t om = (int64_t)(excl & 0xFFFFF), ofl = (int64_t)((excl >> 20) & 0xFFFFF),
                      ol = (int64_t)((excl >> 40) & 0xFFFFF);
        if (t < total && f) {
            double v[9];
            int64_t id, rem;
            soa_load(a.stage, t, v, id, rem);
            if (f & 2) {
                const int64_t dst = base[0] + om;
                if (dst < a.drain_capacity) soa_store(a.drain, dst, v, id, rem);
                else if (a.err) atomicOr(a.err, LCB_DEVERR_CAPACITY);
            } else if (f & 4) {
                const int64_t dst = base[1] + ofl;
                if (dst < a.fell_capacity) soa_store(a.fout, dst, v, id, rem);
                else if (a.err) atomicOr(a.err, LCB_DEVERR_CAPACITY);
            } else if ((f & 1) && a.lost.id) {
                const int64_t dst = base[2] + ol;
                if (dst < a.lost_capacity) soa_store(a.lost, dst, v, id, rem);
                else if (a.err) atomicOr(a.err, LCB_DEVERR_CAPACITY);
            }
        }
        __syncthreads();
        if (tid == CMP_THREADS - 1) {
            const unsigned long long tot = excl + mine;
            base[0] += (long long)(tot & 0xFFFFF);
            base[1] += (long long)((tot >> 20) & 0xFFFFF);
            base[2] += (long long)((tot >> 40) & 0xFFFFF);
        }
        __syncthreads();
    }
    if (tid == 0) {
        *a.drain_count = base[0] < a.drain_capacity ? base[0] : a.drain_capacity;
        *a.fell_out_count = base[1] < a.fell_capacity ? base[1] : a.fell_capacity;
        if (a.lost_count) *a.lost_count = base[2] < a.lost_capacity ? base[2] : a.lost_capacity;
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
    PushParams P;
    P.xi_step = xi_step; P.r_max = r_max; P.h = h; P.N = grid_steps;
    P.xi_k = (double)beam_layer_idx * (-xi_step);
    P.xi_k1 = (double)(beam_layer_idx + 1) * (-xi_step);
    k_beam_move<<<grid_for(n, 128), 128, 0, as_stream(stream)>>>(
        n, P, q_m, dt, F, remaining_steps, id, x, y, xi, px, py, pz, flags, err);
    LCB_LAUNCH_CHECK("k_beam_move");
    return LCB_OK;
}

static bool soa_ok(const lcb_beam_soa &s)
{
    return s.xi && s.x && s.y && s.px && s.py && s.pz && s.q_m && s.q_norm && s.id &&
           s.dt && s.remaining_steps;
}

extern "C" int lcb_beam_step(const lcb_beam_step_args *a, void *stream)
{
    LCB_REQUIRE(a, "args is NULL");
    LCB_REQUIRE(a->grid_steps >= 5 && a->h > 0 && a->xi_step > 0, "bad grid parameters");
    LCB_REQUIRE(a->layout_begin >= 0 && a->layout_end >= a->layout_begin &&
                a->move_begin >= 0 && a->move_end >= a->move_begin, "bad layer slices");
    LCB_REQUIRE(a->substep_energy > 0, "beam-substepping-energy must be > 0");
    LCB_REQUIRE(a->fell_in_count && a->fell_out_count && a->drain_count && a->stage_flags,
                "device counters / flags are NULL");
    LCB_REQUIRE(a->fields_k && a->fields_k1, "fields are NULL");
    LCB_REQUIRE(soa_ok(a->source) && soa_ok(a->fell_in) && soa_ok(a->fell_out) &&
                soa_ok(a->drain) && soa_ok(a->stage), "beam arrays are NULL");
    LCB_REQUIRE(a->move_end - a->move_begin <= a->stage_capacity,
                "stage capacity %lld < fresh layer %lld", (long long)a->stage_capacity,
                (long long)(a->move_end - a->move_begin));
    LCB_REQUIRE(a->ro0 && a->ro1, "density planes are NULL");
    cudaStream_t st = as_stream(stream);
    const int N = a->grid_steps;
    StepArgs s;
    s.src = a->source; s.fin = a->fell_in; s.stage = a->stage;
    s.move_begin = a->move_begin; s.n_fresh = a->move_end - a->move_begin;
    s.fell_in_count = a->fell_in_count;
    s.stage_capacity = a->stage_capacity;
    s.flags = a->stage_flags;
    s.e_sub = a->substep_energy; s.time_step = a->time_step;
    s.P.xi_step = a->xi_step; s.P.r_max = a->r_max; s.P.h = a->h; s.P.N = N;
    s.P.xi_k = (double)(a->layer_idx - 1) * (-a->xi_step);
    s.P.xi_k1 = (double)(a->layer_idx) * (-a->xi_step);
    for (int c = 0; c < 6; c++) {
        s.F.k[c] = a->fields_k->f[c];
        s.F.k1[c] = a->fields_k1->f[c];
        LCB_REQUIRE(s.F.k[c] && s.F.k1[c], "field plane %d is NULL", c);
    }
    s.clear = a->ro1;
    s.clear_n = (int64_t)N * N;
    s.err = a->err;
    k_beam_push_stage<<<2 * sm_count(), 128, 0, st>>>(s);
    LCB_LAUNCH_CHECK("k_beam_push_stage");
    CompactArgs c;
    c.stage = a->stage; c.drain = a->drain; c.fout = a->fell_out; c.lost = a->lost;
    c.flags = a->stage_flags;
    c.n_fresh = s.n_fresh; c.fell_in_count = a->fell_in_count;
    c.stage_capacity = a->stage_capacity;
    c.drain_count = a->drain_count; c.fell_out_count = a->fell_out_count;
    c.lost_count = a->lost.id ? a->lost_count : nullptr;
    c.drain_capacity = a->drain_capacity; c.fell_capacity = a->fell_capacity;
    c.lost_capacity = a->lost_capacity;
    c.err = a->err;
    k_beam_compact<<<1, CMP_THREADS, 0, st>>>(c);
    LCB_LAUNCH_CHECK("k_beam_compact");
    // the layout reads only the source and ro1 was cleared by the push grid
    if (a->layout_end > a->layout_begin) {
        const int64_t n = a->layout_end - a->layout_begin, o = a->layout_begin;
        k_beam_deposit<<<grid_for(n, 128), 128, 0, st>>>(
            n, N, a->h, a->xi_step, -a->xi_step * (double)a->layout_idx,
            a->source.x + o, a->source.y + o, a->source.xi + o, a->source.q_norm + o,
            a->ro0, a->ro1, a->err);
        LCB_LAUNCH_CHECK("k_beam_deposit");
    }
    return LCB_OK;
}
