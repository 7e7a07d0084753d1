/* A plain C (C11) client of the fbls_b200 C ABI: it includes the public
 * header as C, links the built library the way a foreign host does (cgo,
 * Rust's extern "C", JNI or a C program), and calls the entry points that
 * run on the host: the version string, the period grid (count query, fill,
 * short buffer), the segment edges and detrending windows of the
 * reference's own test cases (src/prep/curve.rs:609-622), the prepared
 * family state of the noise-model test's series (curve.rs:636-661) and its
 * error paths (the reference's message; a null array), the refusal of an
 * infinite period grid, and context creation, which
 * without a visible CUDA device must fail with FBLS_ERR_CUDA and a NULL
 * context rather than abort. Prints one JSON object; exits nonzero when a
 * check failed. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fbls_b200.h"

static int fails = 0;

#define CHECK(cond)                                                        \
    do {                                                                   \
        if (!(cond)) {                                                     \
            fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #cond); \
            fails++;                                                       \
        }                                                                  \
    } while (0)

int main(void) {
    /* version */
    const char* version = fbls_version();
    CHECK(version != NULL && strncmp(version, "fbls_b200", 9) == 0);

    /* period grid (grid.rs:34-42's arguments) */
    const int64_t count = fbls_period_grid(0.5, 20.0, 50.0, 0.02, 3.0, NULL, 0);
    CHECK(count > 2);
    double* grid = (double*)malloc((size_t)(count > 0 ? count : 1) * sizeof(double));
    CHECK(grid != NULL);
    int64_t short_count = -1;
    if (grid && count > 2) {
        grid[0] = -1.0;
        short_count = fbls_period_grid(0.5, 20.0, 50.0, 0.02, 3.0, grid, count - 1);
        CHECK(short_count == count);
        CHECK(grid[0] == -1.0); /* not written: capacity too small */
        CHECK(fbls_period_grid(0.5, 20.0, 50.0, 0.02, 3.0, grid, count) == count);
        CHECK(grid[0] == 0.5 && grid[count - 1] == 20.0);
        for (int64_t i = 1; i < count; i++) CHECK(50.0 * (grid[i] / grid[i - 1] - 1.0) <= 0.02 / 3.0 * (1.0 + 1e-9));
    }

    /* segment edges and detrending windows (curve.rs:609-622) */
    const double t5[5] = {0.0, 1.0, 2.0, 10.0, 10.2};
    const double want_edges[5] = {0.0, 1.0, 0.0, 0.0, 0.0};
    double edges[5];
    CHECK(fbls_segment_edges(t5, 5, 1.5, edges) == FBLS_OK);
    for (int i = 0; i < 5; i++) CHECK(edges[i] == want_edges[i]);
    CHECK(fbls_segment_edges(NULL, 5, 1.5, edges) == FBLS_ERR_ARGUMENT);
    const double d5[5] = {0.5 / 24.0, 1.0 / 24.0, 2.0 / 24.0, 12.0 / 24.0, 40.0 / 24.0};
    double windows[5];
    uint32_t family[5], n_windows = 0;
    CHECK(fbls_detrending_windows(d5, 5, 0.4, 3.0, 3.5, windows, family, &n_windows) == FBLS_OK);
    CHECK(n_windows == 3);
    if (n_windows == 3) CHECK(windows[0] == 0.4 && windows[1] == 1.5 && windows[2] == 3.5);
    CHECK(family[0] == 0 && family[1] == 0 && family[2] == 0 && family[3] == 1 && family[4] == 2);

    /* prepared family state of the noise-model test's series (curve.rs:636-661) */
    enum { N = 500 };
    static double t[N], f[N], e[N], to[N], vo[N], wo[N];
    for (int i = 0; i < N; i++) {
        t[i] = 1000.0 + i * 0.01;
        f[i] = 1.0 + 3e-3 * sin(i * 1.7);
        e[i] = 1e-3;
    }
    const double durations[2] = {0.05, 0.1};
    double scalars[5], rho[2];
    char error[128] = "";
    uint32_t n_out = 0;
    CHECK(fbls_family_state(t, f, e, N, durations, 2, 1, &n_out, to, vo, wo, scalars, rho, error, sizeof error) ==
          FBLS_OK);
    CHECK(n_out == N);
    CHECK(to[0] == 0.0 && scalars[1] == 1000.0); /* times relative to the origin */
    CHECK(scalars[0] > 0.0 && scalars[3] > 2.0);  /* baseline_norm; inflation of unit-scale differences */
    CHECK(rho[0] >= 1.0 && rho[1] >= 1.0);
    int data_status = fbls_family_state(t, f, e, 2, durations, 2, 1, &n_out, to, vo, wo, scalars, rho, error,
                                        sizeof error);
    CHECK(data_status == FBLS_ERR_DATA);
    CHECK(strcmp(error, "insufficient usable observations") == 0);
    char null_error[32] = "";
    CHECK(fbls_family_state(NULL, f, e, N, durations, 2, 1, &n_out, to, vo, wo, scalars, rho, null_error,
                            sizeof null_error) == FBLS_ERR_ARGUMENT);
    CHECK(strcmp(null_error, "null argument") == 0);
    CHECK(fbls_period_grid(0.0, 20.0, 50.0, 0.02, 3.0, NULL, 0) == -1); /* infinite grid */

    /* context creation */
    int status = -1;
    fbls_ctx* ctx = fbls_create(0, &status);
    const int device = ctx != NULL;
    if (ctx) {
        CHECK(status == FBLS_OK);
        CHECK(fbls_last_error(ctx) != NULL);
        fbls_destroy(ctx);
    } else {
        CHECK(status == FBLS_ERR_CUDA);
    }
    CHECK(strcmp(fbls_last_error(NULL), "null context") == 0);

    printf("{\"fails\": %d, \"version\": \"%s\", \"grid_count\": %lld, \"device\": %d, \"create_status\": %d, "
           "\"data_error\": \"%s\", \"n_out\": %u}\n",
           fails, version ? version : "", (long long)count, device, status, error, n_out);
    free(grid);
    return fails != 0;
}
