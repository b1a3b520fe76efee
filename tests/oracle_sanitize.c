/* oracle_sanitize.c -- drives the FP64 oracle (oracle/ippi_oracle.c) through
 * its scenes under AddressSanitizer and UndefinedBehaviorSanitizer: the flat
 * plate with each collision, the channel with an IB cylinder (Peskin and
 * bilinear kernels, two direct-forcing passes), solid nodes, and the
 * alternative closures.  Exit status 0 when every call succeeded; the
 * sanitizers abort on the first invalid access or undefined operation. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ippi_oracle.h"

static orc_params params(int nx, int ny, int coll, int bc, int les, int kern)
{
    orc_params p;
    memset(&p, 0, sizeof p);
    p.nx = nx;
    p.ny = ny;
    p.collision = coll;
    p.bc_set = bc;
    p.les_model = les;
    p.tau0 = 0.56;
    p.cs = 0.1;
    p.u_in = 0.05;
    p.rho0 = 1.0;
    p.plate_x0 = nx / 3;
    p.avg_start = 5;
    p.delta_kernel = kern;
    p.mdf_iters = 2;
    return p;
}

static int drain(orc* s, int nx, int ny)
{
    size_t nn = (size_t)nx * ny;
    double* buf = malloc(9 * nn * sizeof(double));
    double f[4], m = 0;
    if (!buf) return 1;
    for (int k = 0; k <= 9; k++) orc_get(s, k, buf);
    orc_forces(s, f, &m);
    free(buf);
    return !(m > 0);
}

int main(void)
{
    int bad = 0;
    for (int coll = 0; coll < 3; coll++) {  /* flat plate */
        orc_params p = params(96, 40, coll, 0, 1, 1);
        orc* s = orc_create(&p);
        orc_init_macros(s, NULL, NULL, NULL);
        bad |= orc_step(s, 12, 1) != 0;
        bad |= drain(s, p.nx, p.ny);
        orc_destroy(s);
    }
    for (int kern = 0; kern < 2; kern++) {  /* channel + IB cylinder */
        orc_params p = params(120, 48, 1, 1, 1, kern);
        orc* s = orc_create(&p);
        double xy[2 * 38];
        for (int m = 0; m < 38; m++) {
            xy[2 * m] = 40.3 + 6.0 * sin(2 * M_PI * m / 38);
            xy[2 * m + 1] = 24.1 + 6.0 * cos(2 * M_PI * m / 38);
        }
        orc_init_macros(s, NULL, NULL, NULL);
        bad |= orc_set_markers(s, 38, xy, NULL, NULL, NULL) != 0;
        bad |= orc_step(s, 12, 1) != 0;
        bad |= drain(s, p.nx, p.ny);
        orc_destroy(s);
    }
    {  /* channel + solid cylinder, then the closures 4-6 */
        orc_params p = params(120, 48, 2, 1, 1, 1);
        orc* s = orc_create(&p);
        unsigned char* solid = calloc((size_t)p.nx * p.ny, 1);
        for (int y = 0; y < p.ny; y++)
            for (int x = 0; x < p.nx; x++) solid[y * p.nx + x] = hypot(x - 40.0, y - 24.0) < 6.0;
        orc_init_macros(s, NULL, NULL, NULL);
        bad |= orc_set_solid(s, solid) != 0;
        bad |= orc_step(s, 12, 1) != 0;
        double fs[2];
        orc_solid_force(s, fs);
        bad |= drain(s, p.nx, p.ny);
        orc_destroy(s);
        for (int les = 4; les <= 6; les++) {
            orc_params q = params(120, 48, 1, 1, les, 1);
            orc* t = orc_create(&q);
            double* d = malloc((size_t)q.nx * q.ny * sizeof(double));
            for (int y = 0; y < q.ny; y++)
                for (int x = 0; x < q.nx; x++) d[y * q.nx + x] = fabs(hypot(x - 40.0, y - 24.0) - 6.0) + 0.5;
            orc_init_macros(t, NULL, NULL, NULL);
            if (les == 6) bad |= orc_set_wall_distance(t, d) != 0;
            bad |= orc_step(t, 8, 1) != 0;
            bad |= drain(t, q.nx, q.ny);
            free(d);
            orc_destroy(t);
        }
        free(solid);
    }
    printf(bad ? "oracle sanitizer run: a call failed\n" : "oracle sanitizer run: ok\n");
    return bad;
}
