/*
 * CPU restatement of MATLAB's pchip(x, y), the B-H table builder that
 * src/MaterialLib.m:117 calls. TEST INFRASTRUCTURE ONLY (results to compare the GPU with).
 *
 * MATLAB is not installed, so this follows MATLAB's published algorithm
 * (Fritsch-Carlson monotone slopes: interior slope = scaled weighted harmonic
 * mean of neighbouring secants when they share a sign, else 0; end slopes by
 * the shape-preserving one-sided three-point rule; Hermite coefficients
 * highest power first). Bits versus MATLAB are unpinned; tests cross-check
 * this against scipy.interpolate.PchipInterpolator.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>

static double sgn(double v) { return (v > 0) - (v < 0); }

static double end_slope(double h1, double h2, double d1, double d2) {
    double d = ((2 * h1 + h2) * d1 - h1 * d2) / (h1 + h2);
    if (sgn(d) != sgn(d1))
        d = 0;
    else if (sgn(d1) != sgn(d2) && fabs(d) > fabs(3 * d1))
        d = 3 * d1;
    return d;
}

int oracle_pchip(const double *x, const double *y, int64_t n, double *coefs) {
    if (n < 2) return -1;
    double *h = (double *)malloc((size_t)n * sizeof(double));
    double *del = (double *)malloc((size_t)n * sizeof(double));
    double *d = (double *)calloc((size_t)n, sizeof(double));
    if (!h || !del || !d) {
        free(h);
        free(del);
        free(d);
        return -1;
    }
    for (int64_t k = 0; k + 1 < n; k++) {
        h[k] = x[k + 1] - x[k];
        if (!(h[k] > 0)) {
            free(h);
            free(del);
            free(d);
            return -2;
        }
        del[k] = (y[k + 1] - y[k]) / h[k];
    }
    if (n == 2) {
        d[0] = d[1] = del[0];
    } else {
        for (int64_t k = 0; k + 2 < n; k++) {
            if (sgn(del[k]) * sgn(del[k + 1]) > 0) {
                double hs = h[k] + h[k + 1];
                double w1 = (h[k] + hs) / (3 * hs);
                double w2 = (hs + h[k + 1]) / (3 * hs);
                double a = fabs(del[k]), b = fabs(del[k + 1]);
                double dmax = a > b ? a : b, dmin = a < b ? a : b;
                d[k + 1] = dmin / (w1 * (del[k] / dmax) + w2 * (del[k + 1] / dmax));
            }
        }
        d[0] = end_slope(h[0], h[1], del[0], del[1]);
        d[n - 1] = end_slope(h[n - 2], h[n - 3], del[n - 2], del[n - 3]);
    }
    for (int64_t k = 0; k + 1 < n; k++) {
        double a = (del[k] - d[k]) / h[k];
        double b = (d[k + 1] - del[k]) / h[k];
        coefs[4 * k + 0] = (b - a) / h[k];
        coefs[4 * k + 1] = 2 * a - b;
        coefs[4 * k + 2] = d[k];
        coefs[4 * k + 3] = y[k];
    }
    free(h);
    free(del);
    free(d);
    return 0;
}
