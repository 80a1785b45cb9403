/* A C99 caller of the C ABI (include/ctfp.h): one plan, spectral tables, a
 * forward through host buffers, the results printed one per line.  Built and
 * run by tests/test_capi.py; its output is compared with the Python host
 * mirror's on the same inputs. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "ctfp.h"

#define CHECK(call)                                                            \
    do {                                                                       \
        ctfp_status s_ = (call);                                               \
        if (s_ != CTFP_OK) {                                                   \
            fprintf(stderr, "%s: %d: %s\n", #call, (int)s_, ctfp_last_error_string()); \
            return 1;                                                          \
        }                                                                      \
    } while (0)

int main(void)
{
    ctfp_geometry g = {0};
    g.pNumX = 16; g.pNumY = 14; g.pNumZ = 12;
    g.pLengthX = 16.0f; g.pLengthY = 14.0f; g.pLengthZ = 12.0f;
    g.projNum = 4; g.dNumU = 20; g.dNumV = 15; g.dSize = 1.6f;
    g.sod = 300.0f; g.sdd = 450.0f; g.rotatedDirection = 1;
    const size_t nvox = 16 * 14 * 12, nray = 4 * 20 * 15, npix = 20 * 15;

    float* rho = malloc(nvox * sizeof(float));
    for (size_t k = 0; k < nvox; k++) rho[k] = 0.5f + (float)(k % 7) * 0.25f;
    const float spectrum[3] = {0.2f, 0.5f, 0.3f};
    const float mu[3] = {0.040f, 0.025f, 0.018f};  /* [E][M], M = 1 */

    ctfp_plan* plan = NULL;
    CHECK(ctfp_plan_create(&g, 1, CTFP_INTERP_TRILINEAR, 0, &plan));
    CHECK(ctfp_set_spectral_tables(plan, 3, spectrum, mu, NULL, CTFP_GRID_NONE, NULL, 1000.0f));
    float* I = malloc(nray * sizeof(float));
    float* A = malloc(nray * sizeof(float));
    float* I0 = malloc(npix * sizeof(float));
    const float* vols[1] = {rho};
    CHECK(ctfp_forward_host(plan, vols, I, A, I0, NULL));
    CHECK(ctfp_plan_destroy(plan));
    for (size_t r = 0; r < nray; r++) {
        if (!(I[r] > 0.0f) || !(I[r] <= I0[r % npix] * 1.000001f) || !isfinite(A[r])) {
            fprintf(stderr, "ray %zu: I %g IAbsorb %g I0 %g\n", r, I[r], A[r], I0[r % npix]);
            return 2;
        }
        printf("%.9g %.9g\n", I[r], A[r]);
    }
    free(rho); free(I); free(A); free(I0);
    return 0;
}
