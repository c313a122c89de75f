/*
 * Plain-C replay harness for the MEX-compatible entry point, for machines
 * without MATLAB: reads the seventeen assemble_jacobian_kernel_mex inputs as
 * raw little-endian float64 files from a directory (names below; the element,
 * node and dof counts follow from the file sizes), calls mag_mex_jacobian, and
 * writes I, J, V, R_idx, R_val as raw float64 files into an output directory.
 *
 *   replay <input_dir> <output_dir> [calcJ=1]
 *
 * Input files: P T Dofs Signs Tags SolA Qw CurlRef lin isNon maxB brk coe start
 * cnt coeStart (each "<name>.f64"). magpackage_b200/harness/write_inputs.py
 * writes them from Python; MATLAB writes them with fwrite(fid, x, 'double').
 * Build: cc -O2 -I<repo>/include replay.c -L<repo>/magpackage_b200 -lmagasm -o replay
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "magasm.h"

static double *load(const char *dir, const char *name, long *count) {
    char path[4096];
    snprintf(path, sizeof path, "%s/%s.f64", dir, name);
    FILE *f = fopen(path, "rb");
    if (!f) {
        fprintf(stderr, "cannot open %s\n", path);
        exit(2);
    }
    fseek(f, 0, SEEK_END);
    long bytes = ftell(f);
    fseek(f, 0, SEEK_SET);
    *count = bytes / 8;
    double *p = (double *)malloc(bytes ? (size_t)bytes : 8);
    if (!p || fread(p, 1, (size_t)bytes, f) != (size_t)bytes) {
        fprintf(stderr, "cannot read %s\n", path);
        exit(2);
    }
    fclose(f);
    return p;
}

static void save(const char *dir, const char *name, const double *p, long n) {
    char path[4096];
    snprintf(path, sizeof path, "%s/%s.f64", dir, name);
    FILE *f = fopen(path, "wb");
    if (!f || fwrite(p, 8, (size_t)n, f) != (size_t)n) {
        fprintf(stderr, "cannot write %s\n", path);
        exit(2);
    }
    fclose(f);
}

int main(int argc, char **argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s <input_dir> <output_dir> [calcJ=1]\n", argv[0]);
        return 1;
    }
    int calcj = argc > 3 ? atoi(argv[3]) : 1;
    long nP, nT, nD, nS, nG, nA, nq, nC, nmat, n1, n2, nb, nc, n3, n4, n5;
    double *P = load(argv[1], "P", &nP), *T = load(argv[1], "T", &nT);
    double *Dofs = load(argv[1], "Dofs", &nD), *Signs = load(argv[1], "Signs", &nS);
    double *Tags = load(argv[1], "Tags", &nG), *Sol = load(argv[1], "SolA", &nA);
    double *Qw = load(argv[1], "Qw", &nq), *Curl = load(argv[1], "CurlRef", &nC);
    double *lin = load(argv[1], "lin", &nmat), *isNon = load(argv[1], "isNon", &n1);
    double *maxB = load(argv[1], "maxB", &n2), *brk = load(argv[1], "brk", &nb);
    double *coe = load(argv[1], "coe", &nc), *start = load(argv[1], "start", &n3);
    double *cnt = load(argv[1], "cnt", &n4), *coeStart = load(argv[1], "coeStart", &n5);
    long Nn = nP / 3, Ne = nT / 4;
    if (nD != 6 * Ne || nS != 6 * Ne || nG != Ne || nC != 18 * nq || n1 != nmat || n2 != nmat ||
        n3 != nmat || n4 != nmat || n5 != nmat) {
        fprintf(stderr, "inconsistent input sizes\n");
        return 1;
    }
    long nk = calcj ? 36 * Ne : 0;
    double *I = calloc(nk ? nk : 1, 8), *J = calloc(nk ? nk : 1, 8), *V = calloc(nk ? nk : 1, 8);
    double *Ri = calloc(6 * Ne, 8), *Rv = calloc(6 * Ne, 8);
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    int rc = mag_mex_jacobian(P, Nn, T, Ne, Dofs, Signs, Tags, Sol, nA, Qw, (int)nq, Curl, lin, isNon,
                              maxB, (int)nmat, brk, (int)nb, coe, (int)nc, start, cnt, coeStart, calcj,
                              I, J, V, Ri, Rv);
    clock_gettime(CLOCK_MONOTONIC, &t1);
    if (rc != MAG_OK) {
        fprintf(stderr, "mag_mex_jacobian failed (%d): %s\n", rc, mag_last_error());
        return 3;
    }
    if (nk) {
        save(argv[2], "I", I, nk);
        save(argv[2], "J", J, nk);
        save(argv[2], "V", V, nk);
    }
    save(argv[2], "R_idx", Ri, 6 * Ne);
    save(argv[2], "R_val", Rv, 6 * Ne);
    double sv = 0, sr = 0;
    for (long i = 0; i < nk; i++) sv += V[i];
    for (long i = 0; i < 6 * Ne; i++) sr += Rv[i];
    printf("elements %ld nodes %ld dofs %ld: sum(V)=%.17g sum(R_val)=%.17g in %.3f ms\n", Ne, Nn, nA,
           sv, sr, (t1.tv_sec - t0.tv_sec) * 1e3 + (t1.tv_nsec - t0.tv_nsec) * 1e-6);
    return 0;
}
