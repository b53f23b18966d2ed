/* Exhaustive-by-sampling check of the plain step's division routine (div_rn in
 * 2dradiation_b200/csrc/kernels_plain.cu) against IEEE division: the same
 * operations in host IEEE FP64 (correctly rounded multiply, fma, reciprocal),
 * which is the arithmetic the device performs.  Prints the mismatch count.
 * usage: division_check <samples> <seed> */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static uint64_t sm(uint64_t *s)
{
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double div_rn(double num, double den, double r)
{
    const double an = fabs(num);
    if (an != 0.0 && !(an > 0x1p-900 && an < 0x1p+900))
        return num / den;
    double q = num * r;
    q = fma(fma(-q, den, num), r, q);
    return fma(fma(-q, den, num), r, q);
}

static double bits(uint64_t sign, int64_t exp, uint64_t man)
{
    uint64_t u = (sign << 63) | ((uint64_t)(exp + 1023) << 52) | (man & ((1ull << 52) - 1));
    double d;
    memcpy(&d, &u, 8);
    return d;
}

int main(int argc, char **argv)
{
    long long n = argc > 1 ? atoll(argv[1]) : 1000000;
    uint64_t s = argc > 2 ? strtoull(argv[2], 0, 10) : 1;
    long long bad = 0;
    for (long long k = 0; k < n; k++)
    {
        const uint64_t a = sm(&s), b = sm(&s), c = sm(&s);
        double num, den;
        switch (k & 3)
        {
        case 0: /* the step's range: intensities and sources over 1 + alpha dt (kappaA + kappa0) */
            num = bits(0, (int64_t)(c % 80) - 60, a);
            den = bits(0, (int64_t)((c >> 8) % 12), b);
            break;
        case 1: /* whole admitted range of den, wide range of num */
            num = bits(c >> 63, (int64_t)(c % 1799) - 899, a);
            den = bits(0, (int64_t)((c >> 16) % 100), b);
            break;
        case 2: /* mantissas with long runs of ones or zeros */
            num = bits(0, (int64_t)(c % 40) - 20, (a & 1) ? ~0ull << (a % 52) : ~(~0ull << (a % 52)));
            den = bits(0, (int64_t)((c >> 8) % 8), (b & 1) ? ~0ull << (b % 52) : (b >> 12));
            break;
        default: /* den just above 1 and quotients near representable midpoints */
            den = 1.0 + ldexp((double)(b >> 11), -53 - (int)(c % 20));
            num = bits(0, (int64_t)(c % 30) - 15, a);
            break;
        }
        if (!(den >= 1.0 && den < 0x1p+100))
            continue;
        const double r = 1.0 / den;
        const double q = div_rn(num, den, r), ref = num / den;
        if (memcmp(&q, &ref, 8) != 0)
        {
            if (bad < 5)
                printf("mismatch %a / %a: %a vs %a\n", num, den, q, ref);
            bad++;
        }
    }
    printf("%lld\n", bad);
    return 0;
}
