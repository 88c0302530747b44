// Declustering noise filter of the plasma electrons (the reference's
// lcode/plasma3d/noise_filter.py:82-239), applied after the last particle
// move of an xi step when 'declustering-enabled' is set.  Two kernels on the
// electrons' Ns x Ns lattice; the Gaussian averaging between them is a
// Fourier-space multiply done by the host with cuFFT (torch.fft).
#include "common.cuh"

namespace lcb {

// Offset inhomogeneity along one lattice direction (noise_filter.py:52-73):
// a point minus the mean of its two neighbours, one-sided second
// differences at the two ends, and 0 wherever a point of the stencil has an
// offset of exactly 0.  d points to the line, element k at d[k * s].
__device__ __forceinline__ double inhomogeneity(const double *d, int64_t s, int j, int n)
{
    if (j > 0 && j < n - 1) {
        const double a = d[(j - 1) * s], c = d[j * s], b = d[(j + 1) * s];
        return (c != 0 && a != 0 && b != 0) ? c - (a + b) / 2 : 0.0;
    }
    if (j == 0) {
        const double c0 = d[0], c1 = d[s], c2 = d[2 * s];
        return (c0 != 0 && c1 != 0 && c2 != 0) ? c0 - 2 * c1 + c2 : 0.0;
    }
    const double c0 = d[(n - 1) * s], c1 = d[(n - 2) * s], c2 = d[(n - 3) * s];
    return (c0 != 0 && c1 != 0 && c2 != 0) ? c0 - 2 * c1 + c2 : 0.0;
}

// dx_inhom, dy_inhom: the mean of the two directions' inhomogeneities of
// x_offt and y_offt (noise_filter.py:123-124).
__global__ void k_decl_inhomogeneity(int n, const double *__restrict__ xo,
                                     const double *__restrict__ yo, double *dx, double *dy)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * n) return;
    const int i = (int)(t / n), j = (int)(t % n);
    const int64_t row = (int64_t)i * n;
    dx[t] = (inhomogeneity(xo + row, 1, j, n) + inhomogeneity(xo + j, n, i, n)) / 2;
    dy[t] = (inhomogeneity(yo + j, n, i, n) + inhomogeneity(yo + row, 1, j, n)) / 2;
}

struct DeclPoint {
    double cx, cy, lim, fx, fy;
};

// Chaotic displacement (inhomogeneity less its average), the limiter
// 1 - d^2 / d_max^2 (0 beyond d_max) and the restoring force at one point
// (noise_filter.py:164-184), in the reference's operation order.
__device__ __forceinline__ DeclPoint decl_point(const lcb_declustering_args &a, int64_t t)
{
    DeclPoint p;
    p.cx = a.dx_inhom[t] - a.dx_average[t];
    p.cy = a.dy_inhom[t] - a.dy_average[t];
    const double d = p.cx * p.cx + p.cy * p.cy, m2 = a.limit * a.limit;
    p.lim = d < m2 ? 1 - d / m2 : 0.0;
    p.fx = -a.force * p.cx * p.lim;
    p.fy = -a.force * p.cy * p.lim;
    return p;
}

// Momentum kicks (noise_filter.py:218-232): each point receives half of its
// own force along each lattice direction in which it is interior, minus a
// quarter of each interior neighbour's, and the damping of the change of
// its chaotic displacement.  Gathered per point: no atomics.
__global__ void k_decl_apply(lcb_declustering_args a)
{
    const int n = a.n;
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * n) return;
    const int i = (int)(t / n), j = (int)(t % n);
    const DeclPoint p = decl_point(a, t);
    const double dxi = a.xi_step;
    double px = a.px[t], py = a.py[t];
    const bool ri = i >= 1 && i <= n - 2, rj = j >= 1 && j <= n - 2;
    // the reference's six slice updates, in its order, for px then py
    double up_x = 0, up_y = 0, dn_x = 0, dn_y = 0, lf_x = 0, lf_y = 0, rt_x = 0, rt_y = 0;
    if (i >= 2) { const DeclPoint q = decl_point(a, t - n); up_x = q.fx; up_y = q.fy; }
    if (i <= n - 3) { const DeclPoint q = decl_point(a, t + n); dn_x = q.fx; dn_y = q.fy; }
    if (j >= 2) { const DeclPoint q = decl_point(a, t - 1); lf_x = q.fx; lf_y = q.fy; }
    if (j <= n - 3) { const DeclPoint q = decl_point(a, t + 1); rt_x = q.fx; rt_y = q.fy; }
    if (ri) px += dxi * p.fx / 2;
    if (i >= 2) px -= dxi * up_x / 4;
    if (i <= n - 3) px -= dxi * dn_x / 4;
    if (rj) px += dxi * p.fx / 2;
    if (j >= 2) px -= dxi * lf_x / 4;
    if (j <= n - 3) px -= dxi * rt_x / 4;
    px -= dxi * a.damping * p.lim * (p.cx - a.dx_chaotic_prev[t]);
    if (ri) py += dxi * p.fy / 2;
    if (i >= 2) py -= dxi * up_y / 4;
    if (i <= n - 3) py -= dxi * dn_y / 4;
    if (rj) py += dxi * p.fy / 2;
    if (j >= 2) py -= dxi * lf_y / 4;
    if (j <= n - 3) py -= dxi * rt_y / 4;
    py -= dxi * a.damping * p.lim * (p.cy - a.dy_chaotic_prev[t]);
    a.px[t] = px;
    a.py[t] = py;
    a.dx_chaotic[t] = p.cx;
    a.dy_chaotic[t] = p.cy;
}

}  // namespace lcb

using namespace lcb;

extern "C" int lcb_declustering_inhomogeneity(int n, const double *x_offt, const double *y_offt,
                                              double *dx_inhom, double *dy_inhom, void *stream)
{
    LCB_REQUIRE(n >= 3, "lattice side %d < 3", n);
    LCB_REQUIRE(x_offt && y_offt && dx_inhom && dy_inhom, "NULL pointer");
    const int64_t nn = (int64_t)n * n;
    k_decl_inhomogeneity<<<(unsigned)((nn + 255) / 256), 256, 0, as_stream(stream)>>>(
        n, x_offt, y_offt, dx_inhom, dy_inhom);
    LCB_LAUNCH_CHECK("k_decl_inhomogeneity");
    return LCB_OK;
}

extern "C" int lcb_declustering_apply(const lcb_declustering_args *a, void *stream)
{
    LCB_REQUIRE(a, "args is NULL");
    LCB_REQUIRE(a->n >= 3, "lattice side %d < 3", a->n);
    LCB_REQUIRE(a->limit > 0, "declustering-limit must be > 0");
    LCB_REQUIRE(a->dx_inhom && a->dy_inhom && a->dx_average && a->dy_average &&
                a->dx_chaotic_prev && a->dy_chaotic_prev && a->px && a->py &&
                a->dx_chaotic && a->dy_chaotic, "NULL pointer");
    LCB_REQUIRE(a->dx_chaotic != a->dx_chaotic_prev && a->dy_chaotic != a->dy_chaotic_prev,
                "the chaotic displacements are written, the previous ones read: "
                "they must be different arrays");
    const int64_t nn = (int64_t)a->n * a->n;
    k_decl_apply<<<(unsigned)((nn + 255) / 256), 256, 0, as_stream(stream)>>>(*a);
    LCB_LAUNCH_CHECK("k_decl_apply");
    return LCB_OK;
}
