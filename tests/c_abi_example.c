/* A plain C caller of the fftb C ABI (include/fftb.h), the way a C or C++ host of the
 * reference's ffts path would use it: no Python, no torch.  Solves the periodic Poisson
 * problem lap u = f on [0, 2 pi)^3 with f = -14 sin x sin 2y cos 3z (exact solution
 * u = sin x sin 2y cos 3z), checks a forward + normalised backward round trip, and
 * exercises a plan and the error path.  Prints one line per check; exit status 0 when
 * every check passes.  Built and run by tests/test_gpu_c_abi.py. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <cuda_runtime.h>

#include "fftb.h"

#define N 32

static int check(int st, const char *what)
{
    if (st != FFTB_SUCCESS) {
        printf("FAIL %s: %s (%s)\n", what, fftb_status_string(st), fftb_last_error_message());
        return 1;
    }
    return 0;
}

int main(void)
{
    const size_t n = (size_t)N * N * N, nc = (size_t)N * N * (N / 2 + 1);
    float *h = (float *)malloc(n * sizeof(float)), *u = (float *)malloc(n * sizeof(float));
    const double pi = 3.14159265358979323846;
    for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y)
            for (int z = 0; z < N; ++z) {
                const double gx = 2 * pi * x / N, gy = 2 * pi * y / N, gz = 2 * pi * z / N;
                h[((size_t)x * N + y) * N + z] = (float)(-14.0 * sin(gx) * sin(2 * gy) * cos(3 * gz));
            }
    float *d_f = NULL, *d_u = NULL;
    void *d_spec = NULL;
    if (cudaMalloc((void **)&d_f, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&d_u, n * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&d_spec, nc * 2 * sizeof(float)) != cudaSuccess) {
        printf("FAIL cudaMalloc\n");
        return 1;
    }
    cudaMemcpy(d_f, h, n * sizeof(float), cudaMemcpyHostToDevice);

    int bad = 0;
    fftb_ffts obj = NULL;
    bad |= check(fftb_ffts_create(FFTB_F32, N, N, N, 0, FFTB_4D_PENCIL, &obj), "fftb_ffts_create");
    if (bad) return 1;
    int dim = 0;
    bad |= check(fftb_ffts_dimension(obj, &dim), "fftb_ffts_dimension");
    printf("dimension %d (library %s)\n", dim, fftb_version());

    /* Poisson: lap u = f (sign -1) */
    bad |= check(fftb_ffts_poisson(obj, d_f, d_u, -1.0), "fftb_ffts_poisson");
    cudaMemcpy(u, d_u, n * sizeof(float), cudaMemcpyDeviceToHost);
    double num = 0, den = 0;
    for (size_t i = 0; i < n; ++i) {
        const double ex = -h[i] / 14.0;
        num += (u[i] - ex) * (u[i] - ex);
        den += ex * ex;
    }
    const double perr = sqrt(num / den);
    printf("poisson rel-L2 vs the exact solution %.3e\n", perr);
    if (!(perr < 1e-5)) bad = 1;

    /* forward + normalised backward round trip */
    bad |= check(fftb_ffts_forward(obj, d_f, d_spec), "fftb_ffts_forward");
    bad |= check(fftb_ffts_backward_normalized(obj, d_spec, d_u), "fftb_ffts_backward_normalized");
    cudaMemcpy(u, d_u, n * sizeof(float), cudaMemcpyDeviceToHost);
    num = den = 0;
    for (size_t i = 0; i < n; ++i) {
        num += (u[i] - h[i]) * (u[i] - h[i]);
        den += (double)h[i] * h[i];
    }
    const double rerr = sqrt(num / den);
    printf("round trip rel-L2 %.3e\n", rerr);
    if (!(rerr < 1e-6)) bad = 1;

    /* a cufft::fft-style plan: batched 1D C2C of a prime length (chirp-z pass) */
    long long len[1] = {17};
    fftb_plan plan = NULL;
    size_t work = 0;
    bad |= check(fftb_plan_create(FFTB_C2CF, FFTB_F32, 1, len, NULL, 1, 17, NULL, 1, 17, 4, &plan, &work),
                 "fftb_plan_create");
    bad |= check(fftb_exec(plan, d_spec, d_spec), "fftb_exec");
    bad |= check(fftb_plan_destroy(plan), "fftb_plan_destroy");

    /* the error path: init twice has no C form, but a wrong direction is rejected */
    int st = fftb_plan_create(99, FFTB_F32, 1, len, NULL, 1, 17, NULL, 1, 17, 1, &plan, &work);
    printf("invalid direction -> %s\n", fftb_status_string(st));
    if (st != FFTB_ERROR_INVALID_VALUE) bad = 1;

    bad |= check(fftb_ffts_destroy(obj), "fftb_ffts_destroy");
    cudaFree(d_f);
    cudaFree(d_u);
    cudaFree(d_spec);
    free(h);
    free(u);
    printf(bad ? "FAILED\n" : "ok\n");
    return bad;
}
