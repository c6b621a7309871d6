/* Checks the division-by-constant used by the cost kernels (div_2pi, div_7
 * in cuphu_b200/csrc/cost.cu) against IEEE division for every float of the
 * ranges the kernels send it (stride 1 = exhaustive).  Prints one line per
 * constant: the number of inputs checked and of mismatches. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static float as_float(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }

/* q0 = RN(x zc); r = x - q0 c (fma); q = RN(q0 + r zc) */
static float div_const(float x, float c, float zc)
{
    float q0 = x * zc;
    float r = fmaf(-q0, c, x);
    return fmaf(r, zc, q0);
}

int main(int argc, char **argv)
{
    uint32_t stride = argc > 1 ? (uint32_t)strtoul(argv[1], 0, 10) : 1u;
    const float two_pi = 6.28318548202514648f;
    const float zc_2pi = 0x1.45f306p-3f, zc_7 = 0x1.24924ap-3f;
    /* the constants are RN(1/c) */
    if ((float)(1.0 / (double)two_pi) != zc_2pi || (float)(1.0 / 7.0) != zc_7) {
        printf("constant mismatch\n");
        return 2;
    }
    long n2 = 0, bad2 = 0, n7 = 0, bad7 = 0;
    for (uint64_t b = 0; b <= 0xffffffffull; b += stride) {
        float x = as_float((uint32_t)b);
        float a = fabsf(x);
        /* div_2pi's fast path: 2^-104 <= |x| <= 6.6 */
        if (a >= 0x1p-104f && a <= 6.6f) {
            float q = div_const(x, two_pi, zc_2pi), ref = x / two_pi;
            ++n2;
            if (memcmp(&q, &ref, 4)) ++bad2;
        }
        /* div_7: |x| <= 3.6, any x but -0 */
        if (a <= 3.6f && !(x == 0.0f && signbit(x))) {
            float q = div_const(x, 7.0f, zc_7), ref = x / 7.0f;
            ++n7;
            if (memcmp(&q, &ref, 4)) ++bad7;
        }
    }
    printf("2pi %ld %ld\n7 %ld %ld\n", n2, bad2, n7, bad7);
    return 0;
}
