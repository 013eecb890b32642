/* Exhaustive check of the division-free Hermite sample parameter
 * (HermTask::sample_t in fastrrt_b200/csrc/frrt_device.cuh): with
 * y = RN(1 / b), q = RN(a y), r = RN(a - q b) (one fused multiply-add, exact)
 * and t = RN(q + r y) (another fused multiply-add), t equals the IEEE
 * quotient RN(a / b) for every 0 <= a <= b <= B.  The device computes the
 * same three correctly rounded operations (__dmul_rn, __fma_rn) and the
 * reciprocal by IEEE division, so this host run decides the claim.
 *
 *   cc -O2 -ffp-contract=off sample_t_check.c -lm && ./a.out [B]
 *
 * Prints the number of pairs checked and of mismatches; exits 1 on any.
 * Built with -DUNCORRECTED it checks the product alone, which the test
 * expects to fail (the check can tell the two apart). */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

int main(int argc, char **argv)
{
    const long B = argc > 1 ? atol(argv[1]) : 16384;
    long pairs = 0, bad = 0;
    for (long b = 1; b <= B; b++) {
        const volatile double span = (double)b;
        const double y = 1.0 / span;
        for (long a = 0; a <= b; a++) {
            const double ak = (double)a;
            const double q = ak * y;
#ifdef UNCORRECTED
            const double t = q;  /* the product alone: not always RN(a / b) */
#else
            const double t = fma(fma(-q, span, ak), y, q);
#endif
            const double want = ak / span;
            pairs++;
            if (t != want) {
                if (bad < 5)
                    printf("mismatch a=%ld b=%ld: %.17g vs %.17g\n", a, b, t, want);
                bad++;
            }
        }
    }
    printf("%ld pairs, %ld mismatches\n", pairs, bad);
    return bad != 0;
}
