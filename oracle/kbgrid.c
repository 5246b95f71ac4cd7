/*
 * CPU restatement of SigPy 0.1.27's Kaiser-Bessel interpolation / gridding
 * loops (the reference's NUFFT, src/toporecon/nufft_backend.py:104-116) --
 * TEST INFRASTRUCTURE / CPU BASELINE ONLY, never linked into the product.
 *
 * Coordinates are already scaled onto the oversampled grid (k * os/n + os//2).
 * Per axis the taps are ceil(k - w/2) .. floor(k + w/2); the window is
 * I0(beta sqrt(1 - d^2)) for |d| = |tap - k| / (w/2) <= 1 (Abramowitz & Stegun
 * 9.8.1 / 9.8.2 for I0), periodic wrap on the grid.  Data are complex64 laid
 * out (batch, points) and (batch, Gz, Gy, Gx).  Weights in double.
 *
 * interpolate: OpenMP over samples.
 * gridding:    OpenMP over z-slabs of the grid; every thread scans all samples
 *              and adds only into its own slab, so the summation order is the
 *              sample order and the result does not depend on the thread count.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

static double i0_as(double x) {
    if (x < 3.75) {
        double t = x / 3.75, t2 = t * t;
        return 1.0 + t2 * (3.5156229 + t2 * (3.0899424 + t2 * (1.2067492 + t2 * (0.2659732 +
               t2 * (0.0360768 + t2 * 0.0045813)))));
    }
    double u = 3.75 / x;
    double poly = 0.39894228 + u * (0.01328592 + u * (0.00225319 + u * (-0.00157565 + u * (0.00916281 +
                  u * (-0.02057706 + u * (0.02635537 + u * (-0.01647633 + u * 0.00392377)))))));
    return exp(x) / sqrt(x) * poly;
}

static double kb(double d, double beta) {
    if (fabs(d) > 1.0) return 0.0;
    return i0_as(beta * sqrt(1.0 - d * d));
}

static int pmod(long a, int n) {
    long r = a % n;
    return (int)(r < 0 ? r + n : r);
}

static void taps(float k, int width, double beta, long* first, double* w) {
    double half = width / 2.0;
    *first = (long)ceil((double)k - half);
    for (int t = 0; t <= width; ++t) w[t] = kb(((double)(*first + t) - (double)k) / half, beta);
}

void kb_interpolate(const float* grid /* (batch, G) complex */, int batch, int gz, int gy, int gx,
                    const float* ks /* (M, 3) */, long M, int width, double beta, float* out /* (batch, M) complex */) {
    const long G = (long)gz * gy * gx;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < M; ++i) {
        double wz[9], wy[9], wx[9];
        long fz, fy, fx;
        taps(ks[3 * i + 0], width, beta, &fz, wz);
        taps(ks[3 * i + 1], width, beta, &fy, wy);
        taps(ks[3 * i + 2], width, beta, &fx, wx);
        for (int b = 0; b < batch; ++b) {
            double re = 0.0, im = 0.0;
            const float* gb = grid + 2 * (long)b * G;
            for (int a = 0; a <= width; ++a) {
                if (wz[a] == 0.0) continue;
                long zo = (long)pmod(fz + a, gz) * gy;
                for (int c = 0; c <= width; ++c) {
                    if (wy[c] == 0.0) continue;
                    double wzy = wz[a] * wy[c];
                    long yo = (zo + pmod(fy + c, gy)) * gx;
                    for (int d = 0; d <= width; ++d) {
                        if (wx[d] == 0.0) continue;
                        double w = wzy * wx[d];
                        long idx = yo + pmod(fx + d, gx);
                        re += w * gb[2 * idx];
                        im += w * gb[2 * idx + 1];
                    }
                }
            }
            out[2 * ((long)b * M + i)] = (float)re;
            out[2 * ((long)b * M + i) + 1] = (float)im;
        }
    }
}

void kb_gridding(const float* vals /* (batch, M) complex */, int batch, const float* ks, long M, int width,
                 double beta, int gz, int gy, int gx, float* grid /* (batch, G) complex, zeroed here */,
                 int nslab) {
    const long G = (long)gz * gy * gx;
    memset(grid, 0, sizeof(float) * 2 * G * batch);
    if (nslab < 1) nslab = 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int s = 0; s < nslab; ++s) {
        const int z0 = (int)((long)gz * s / nslab), z1 = (int)((long)gz * (s + 1) / nslab);
        for (long i = 0; i < M; ++i) {
            double wz[9], wy[9], wx[9];
            long fz, fy, fx;
            taps(ks[3 * i + 0], width, beta, &fz, wz);
            int any = 0;
            for (int a = 0; a <= width; ++a) {
                int z = pmod(fz + a, gz);
                if (wz[a] != 0.0 && z >= z0 && z < z1) any = 1;
            }
            if (!any) continue;
            taps(ks[3 * i + 1], width, beta, &fy, wy);
            taps(ks[3 * i + 2], width, beta, &fx, wx);
            for (int a = 0; a <= width; ++a) {
                int z = pmod(fz + a, gz);
                if (wz[a] == 0.0 || z < z0 || z >= z1) continue;
                for (int c = 0; c <= width; ++c) {
                    if (wy[c] == 0.0) continue;
                    double wzy = wz[a] * wy[c];
                    long yo = ((long)z * gy + pmod(fy + c, gy)) * gx;
                    for (int d = 0; d <= width; ++d) {
                        if (wx[d] == 0.0) continue;
                        double w = wzy * wx[d];
                        long idx = yo + pmod(fx + d, gx);
                        for (int b = 0; b < batch; ++b) {
                            const float* v = vals + 2 * ((long)b * M + i);
                            float* g = grid + 2 * ((long)b * G + idx);
                            g[0] += (float)(w * v[0]);
                            g[1] += (float)(w * v[1]);
                        }
                    }
                }
            }
        }
    }
}
