// Device-side helpers that let a whole xi step of a simulation be captured
// once and replayed: the rigid Gaussian driver evaluated from a step counter
// in device memory, and the on-axis Ez record that advances that counter.
#include "common.cuh"

namespace lcb {

// rho_b(x, y, xi) = A exp(-(x^2 + y^2) / (2 s^2)) (1 + cos(sqrt(pi/2) xi)) / 2
// for -xi_len <= xi <= 0, else 0 -- the rigid driver of the configurations,
// evaluated on the grid (i - N/2) h with the reference's meshgrid orientation
// (beam_calculator.py:158-170: the first index is y, the second x).
__device__ __forceinline__ double gaussian_driver(double A, double s2, double xi_len, double xi,
                                                  double x, double y)
{
    if (!(xi >= -xi_len && xi <= 0)) return 0.0;
    return A * exp(-(x * x + y * y) / (2 * s2)) * (1 + cos(sqrt(M_PI / 2) * xi)) / 2;
}

__global__ void k_rigid_gaussian(int N, double h, double xi_step, double A, double sigma_r,
                                 double xi_len, int64_t first, const int64_t *counter,
                                 double *rho_full, double *rho_prev)
{
    const int64_t c = *counter;
    const int64_t layer = first + c;
    const double xi_full = -(double)layer * xi_step;
    const double xi_prev = -(double)(layer - 1) * xi_step;
    const double s2 = sigma_r * sigma_r;
    const int64_t NN = (int64_t)N * N;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < NN;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / N), j = (int)(t % N);
        const double y = (i - N / 2) * h, x = (j - N / 2) * h;
        rho_full[t] = gaussian_driver(A, s2, xi_len, xi_full, x, y);
        rho_prev[t] = c > 0 ? gaussian_driver(A, s2, xi_len, xi_prev, x, y) : 0.0;
    }
}

__global__ void k_record_axis(const double *plane, int N, int64_t *counter, double *hist,
                              int64_t capacity)
{
    const int64_t c = *counter;
    if (c < capacity) hist[c] = plane[(int64_t)(N / 2) * N + N / 2];
    *counter = c + 1;
}

}  // namespace lcb

using namespace lcb;

extern "C" int lcb_rigid_gaussian(int grid_steps, double h, double xi_step, double amplitude,
                                  double sigma_r, double xi_len, int64_t first_layer,
                                  const int64_t *counter, double *rho_full, double *rho_prev,
                                  void *stream)
{
    LCB_REQUIRE(grid_steps >= 5 && h > 0 && xi_step > 0 && sigma_r > 0, "bad driver arguments");
    LCB_REQUIRE(counter && rho_full && rho_prev, "NULL pointer");
    const int64_t NN = (int64_t)grid_steps * grid_steps;
    const int blocks = (int)((NN + 255) / 256);
    k_rigid_gaussian<<<blocks, 256, 0, as_stream(stream)>>>(
        grid_steps, h, xi_step, amplitude, sigma_r, xi_len, first_layer, counter, rho_full,
        rho_prev);
    LCB_LAUNCH_CHECK("k_rigid_gaussian");
    return LCB_OK;
}

extern "C" int lcb_record_axis(const double *plane, int grid_steps, int64_t *counter,
                               double *history, int64_t capacity, void *stream)
{
    LCB_REQUIRE(plane && counter && history && grid_steps >= 1, "NULL pointer");
    k_record_axis<<<1, 1, 0, as_stream(stream)>>>(plane, grid_steps, counter, history, capacity);
    LCB_LAUNCH_CHECK("k_record_axis");
    return LCB_OK;
}
