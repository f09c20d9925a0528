/*
 * A plain C caller of the FETI4I interface, in the call sequence of the reference's
 * src/app/apitest.cpp: MPI_Init, FETI4ICreateStiffnessMatrix, FETI4IAddElement per element,
 * FETI4ICreateInstance, FETI4ISolve (or, without a GPU, the host preparation only), FETI4IDestroy,
 * MPI_Finalize.  Built with gcc against include/feti4i.h (which includes "mpi.h": the single-process
 * stand-in include/mpi.h) for FETI4I_INT_WIDTH 32 and 64.
 *
 *   feti4i_caller <problem.bin> <out.bin> host|solve
 *
 * problem.bin (little endian): int64 nelem, nodes per element, DOFs per element, DOFs, Dirichlet DOFs,
 * subdomains; int64 nodes[nelem*npe], dofs[nelem*dpe], partition[nelem], dirichlet[ndir];
 * double Ke[nelem*dpe*dpe], rhs[ndofs], dirichlet values[ndir].
 * out.bin: "host": b (dual size) then multipliers of subdomain 0 as double; "solve": the solution.
 */
#include <stdio.h>
#include <stdlib.h>

#include "feti4i.h"
#include "feti4i_ext.h"

static void *read_n(FILE *f, size_t size, size_t n) {
    void *p = malloc(size * (n ? n : 1));
    if (n && fread(p, size, n, f) != n) { fprintf(stderr, "short read\n"); exit(2); }
    return p;
}

static FETI4IInt *ints(const long long *v, long long n) {
    FETI4IInt *o = malloc(sizeof(FETI4IInt) * (n ? n : 1));
    for (long long i = 0; i < n; ++i) o[i] = (FETI4IInt)v[i];
    return o;
}

static int check(const char *where) {
    const char *e = FETI4IGetLastError();
    if (e && e[0]) { fprintf(stderr, "%s: %s\n", where, e); return 1; }
    return 0;
}

int main(int argc, char **argv) {
    if (argc != 4) { fprintf(stderr, "usage: feti4i_caller problem.bin out.bin host|solve\n"); return 2; }
    MPI_Init(&argc, &argv);
    int rank = -1;
    MPI_Comm_rank(MPI_COMM_WORLD, &rank);
    const int solve = argv[3][0] == 's';
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    long long hdr[6];
    if (fread(hdr, sizeof(long long), 6, f) != 6) return 2;
    const long long ne = hdr[0], npe = hdr[1], dpe = hdr[2], nd = hdr[3], ndir = hdr[4], nsub = hdr[5];
    long long *nodes = read_n(f, 8, ne * npe), *dofs = read_n(f, 8, ne * dpe), *part = read_n(f, 8, ne);
    long long *dir = read_n(f, 8, ndir);
    double *Ke = read_n(f, 8, ne * dpe * dpe), *rhs = read_n(f, 8, nd), *dirv = read_n(f, 8, ndir);
    fclose(f);

    FETI4IMatrix K;
    FETI4ICreateStiffnessMatrix(&K, FETI4I_REAL_SYMMETRIC_POSITIVE_DEFINITE, 0);
    if (check("create matrix")) return 1;
    FETI4IInt *in = ints(nodes, ne * npe), *id = ints(dofs, ne * dpe);
    for (long long e = 0; e < ne; ++e)
        FETI4IAddElement(K, FETI4I_VOLUME, (FETI4IInt)npe, in + e * npe, (FETI4IInt)dpe, id + e * dpe,
                         Ke + e * dpe * dpe);
    if (check("add element")) return 1;
    FETI4IInt *ip = ints(part, ne);
    FETI4ISetSubdomainPartition(K, (FETI4IInt)ne, ip);
    FETI4IInt iopts[FETI4I_INTEGER_OPTIONS_SIZE];
    FETI4IReal ropts[FETI4I_REAL_OPTIONS_SIZE];
    FETI4ISetDefaultIntegerOptions(iopts);
    FETI4ISetDefaultRealOptions(ropts);
    iopts[FETI4I_SUBDOMAINS] = (FETI4IInt)nsub;
    iopts[FETI4I_PRECONDITIONER] = 1;
    iopts[FETI4I_VERBOSE_LEVEL] = 0;
    ropts[FETI4I_PRECISION] = 1e-10;
    if (!solve) FETI4ISetExtendedOption(FETI4I_EXT_HOST_ONLY, 1);
    FETI4IInt *l2g = malloc(sizeof(FETI4IInt) * nd), *idir = ints(dir, ndir);
    for (long long i = 0; i < nd; ++i) l2g[i] = (FETI4IInt)i;
    FETI4IInstance inst;
    FETI4ICreateInstance(&inst, K, (FETI4IInt)nd, rhs, l2g, 0, NULL, (FETI4IInt)ndir, idir, dirv, iopts, ropts);
    if (check("create instance")) return 1;
    FILE *o = fopen(argv[2], "wb");
    if (solve) {
        double *u = calloc(nd, sizeof(double));
        FETI4ISolve(inst, (FETI4IInt)nd, u);
        if (check("solve")) return 1;
        fwrite(u, sizeof(double), nd, o);
        free(u);
    } else {
        FETI4IReal stats[FETI4I_STAT_SIZE];
        FETI4IGetStats(inst, FETI4I_STAT_SIZE, stats);
        const long long nl = (long long)stats[FETI4I_STAT_DUAL_SIZE], nk = (long long)stats[FETI4I_STAT_KERNEL_SIZE];
        double *b = calloc(nl, sizeof(double)), *e = calloc(nk, sizeof(double));
        FETI4IGetDualRhs(inst, b, e);
        FETI4IInt info[4];
        FETI4IGetSubdomainInfo(inst, 0, info);
        FETI4IInt *lam = calloc(info[1], sizeof(FETI4IInt));
        FETI4IGetSubdomainMultipliers(inst, 0, lam, NULL, NULL, NULL, NULL);
        if (check("introspection")) return 1;
        fwrite(b, sizeof(double), nl, o);
        for (FETI4IInt r = 0; r < info[1]; ++r) {
            double v = (double)lam[r];
            fwrite(&v, sizeof(double), 1, o);
        }
        FETI4ISetExtendedOption(FETI4I_EXT_HOST_ONLY, 0);
    }
    fclose(o);
    FETI4IDestroy(inst);
    FETI4IDestroy(K);
    MPI_Finalize();
    return rank == 0 ? 0 : 3;
}
