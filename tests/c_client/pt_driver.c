/* pt_driver.c -- a C client of the library that follows the reference's PT driver
 * (src/PT.f90:193-331) through the C-ABI alone: build the mesh (makeChainMesh), draw initial
 * spins, run parallel tempering (sweeps + exchange rounds), read the energies and the
 * temperature-to-replica map, take the winding number of the middle slice of the coldest
 * replica (calculate_winding_number2) and write its spins (write_spins_to_file).
 *
 *   usage: pt_driver L n_temps rounds spins_csv_path
 *   prints one line: "ok <E of each slot...> | <replica of each slot...> | Q"
 *   exits 1 with the library's message on any error. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "ising_gpu.h"

static int check(int st, const char* what) {
    if (st != ISING_OK) {
        fprintf(stderr, "%s failed (%d): %s\n", what, st, ising_last_error());
        exit(1);
    }
    return st;
}

int main(int argc, char** argv) {
    if (argc != 5) {
        fprintf(stderr, "usage: %s L n_temps rounds spins_csv_path\n", argv[0]);
        return 2;
    }
    const int L = atoi(argv[1]), n = atoi(argv[2]), rounds = atoi(argv[3]);
    double a, b, c, ab, bc, ca;
    float frac[36];
    int n_sub = 0;
    check(ising_unit_cell(ISING_CELL_SC, &a, &b, &c, &ab, &bc, &ca, frac, &n_sub), "ising_unit_cell");
    ising_mesh* mesh = NULL;
    check(ising_mesh_create(frac, n_sub, L, L, L, 1.0, 1.0, 1.0, ab, bc, ca, 0.0, 0, n, 0, &mesh), "ising_mesh_create");
    check(ising_spins_init_uniform(mesh, 0x15196u, 0u), "ising_spins_init_uniform");

    /* geometric ladder T_j = Tmin (Tmax/Tmin)^(j/(n-1)) (src/PT.f90:202) */
    double* betas = malloc(sizeof(double) * n);
    for (int j = 0; j < n; ++j) {
        const double T = n > 1 ? 0.1 * pow(15.0, (double)j / (n - 1)) : 0.1;
        betas[j] = 1.0 / T;
    }
    ising_params p;
    check(ising_params_reference(0, -1.0, 0.0, 0.7, 0.0, 0.3, &p), "ising_params_reference");
    p.include_Jp = 0;
    p.dmi_mode = ISING_DMI_BULK;
    ising_pt_options opt = {0};
    opt.seed = 0x15196u;
    opt.move = ISING_MOVE_BALL;
    opt.r = 0.2;
    opt.scheme = ISING_PT_EVEN_ODD;
    ising_pt* pt = NULL;
    check(ising_pt_create(mesh, n, betas, &p, &opt, &pt), "ising_pt_create");
    check(ising_pt_run(pt, 10, rounds), "ising_pt_run");

    double* e = malloc(sizeof(double) * n);
    double* m = malloc(sizeof(double) * 3 * n);
    int* t2r = malloc(sizeof(int) * n);
    check(ising_pt_energies(pt, e, m), "ising_pt_energies");
    check(ising_pt_permutation(pt, t2r), "ising_pt_permutation");
    double q = 0.0;
    check(ising_winding_number(mesh, t2r[0], L / 2, &q), "ising_winding_number");
    check(ising_write_spins_csv(mesh, t2r[0], argv[4], 0, 1, -1), "ising_write_spins_csv");

    printf("ok");
    for (int j = 0; j < n; ++j) printf(" %.9g", e[t2r[j]]);
    printf(" |");
    for (int j = 0; j < n; ++j) printf(" %d", t2r[j]);
    printf(" | %.9g\n", q);

    check(ising_pt_destroy(pt), "ising_pt_destroy");
    check(ising_mesh_destroy(mesh), "ising_mesh_destroy");
    free(betas); free(e); free(m); free(t2r);
    return 0;
}
