/* A C host written against the reference API only (paradmm.h): it builds a
 * circle-packing graph the way packing/host.c does (startG, addNode with the
 * packing operators, initialize_*), seeds the state, calls
 * updateGOpenMP(&G, sweeps, threads) and prints the consensus Z.  The test
 * suite builds this one source twice -- linked against the reference's own
 * library and against libparadmm_b200.so -- and compares the outputs.
 * usage: host_demo N sweeps */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "paradmm.h"

#ifdef PARADMM_B200
int paradmm_last_status(void);
const char *paradmm_last_error_string(void);
#endif

static double u01(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

int main(int argc, char **argv)
{
    const int N = argc > 1 ? atoi(argv[1]) : 60;
    const int sweeps = argc > 2 ? atoi(argv[2]) : 5;
    static double walls[4][4] = {{-1, 0, 0, 0}, {1, 0, 1, 0}, {0, -1, 0, 0}, {0, 1, 0, 1}};
    static double expo = 2.0;
    graph G;
    memset(&G, 0, sizeof G);
    startG(&G, 2);
    for (int i = 0; i < N; ++i)
        for (int j = i + 1; j < N; ++j) {
            int v[4] = {2 * i, 2 * i + 1, 2 * j, 2 * j + 1};
            addNode(&G, disk_collision_variable_radius, NULL, 4, v);
        }
    for (int i = 0; i < N; ++i)
        for (int w = 0; w < 4; ++w) {
            int v[2] = {2 * i, 2 * i + 1};
            addNode(&G, disk_plane_collision_variable_radius, walls[w], 2, v);
        }
    for (int i = 0; i < N; ++i) {
        int v[1] = {2 * i + 1};
        addNode(&G, maximize_sum_of_squared_disk_radii_alpha, &expo, 1, v);
    }
    initialize_RHOS_APHAS(&G, 10.0, 1.0);
    for (int f = 0; f < G.num_opts; ++f)  /* rho 5 on the radius-factor edges */
        if (G.list_of_operators_functions_pointers[f] == maximize_sum_of_squared_disk_radii_alpha)
            for (int k = 0; k < G.operatorix_to_numedges[f]; ++k) G.RHOS[G.operatorix_to_edgelistix[f][k]] = 5.0;
    initialize_X_N_Z_M_U_zeros(&G);
    uint64_t s = 12345;
    for (int i = 0; i < N; ++i) {
        const double cx = u01(&s), cy = u01(&s), r = 0.05 * u01(&s);
        G.Z[4 * i + 0] = cx; G.Z[4 * i + 1] = cy; G.Z[4 * i + 2] = r; G.Z[4 * i + 3] = r;
    }
    for (int e = 0; e < G.num_edges; ++e) {
        const int v = G.edgeix_to_varlistix[e];
        for (int k = 0; k < 2; ++k) {
            G.X[2 * e + k] = G.N[2 * e + k] = G.M[2 * e + k] = G.Z[2 * v + k];
            G.U[2 * e + k] = 0.0;
        }
    }
    updateGOpenMP(&G, sweeps, 4);
#ifdef PARADMM_B200
    if (paradmm_last_status() != 0) {
        fprintf(stderr, "engine error: %s\n", paradmm_last_error_string());
        return 2;
    }
#endif
    for (int v = 0; v < G.num_vars; ++v) printf("%.17g %.17g\n", G.Z[2 * v], G.Z[2 * v + 1]);
    closeG(&G);
    return 0;
}
