// Host-side check of the register DFT kernels of tr_fft.cuh (Dft<R>::run, the
// butterflies every FFT stage applies).  Prints, for each radix R and both
// directions, R input values and the R outputs; the test compares them with
// numpy's FFT.  Built by nvcc as a plain host program (no GPU needed).
#include <cstdio>
#include <cmath>

#include "tr_fft.cuh"

template <int R>
static void check(bool inv) {
    float2 v[R];
    for (int n = 0; n < R; ++n) v[n] = make_float2(std::sin(1.3f * n + R), std::cos(0.7f * n * R + 0.1f));
    std::printf("R %d %d\n", R, inv ? 1 : 0);
    for (int n = 0; n < R; ++n) std::printf("%.9g %.9g\n", v[n].x, v[n].y);
    tr::Dft<R>::run(v, inv);
    for (int n = 0; n < R; ++n) std::printf("%.9g %.9g\n", v[n].x, v[n].y);
}

int main() {
    for (int inv = 0; inv < 2; ++inv) {
        check<2>(inv);
        check<3>(inv);
        check<4>(inv);
        check<5>(inv);
        check<7>(inv);
        check<8>(inv);
        check<10>(inv);
        check<16>(inv);
        check<20>(inv);
    }
    return 0;
}
