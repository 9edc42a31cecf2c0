/* Checker tool, written for this project, that prints the reference's
 * (mrirecon/bart) Kaiser-Bessel window table and roll-off, computed by the
 * reference's own library as a NUFFT plan initialises them. Test
 * infrastructure only.
 *
 *   kbtable [os width [n...]]
 *
 * Prints, one value per line in C99 hex-float notation (exact):
 *   beta <beta as calc_beta returns it>
 *   i0beta <bessel_kb_beta>
 *   kb <i> <table[i]>               for i = 0..kb_size
 *   roll <n> <x> <value>            the roll-off of an n-point axis
 *
 * The table is initialised as nufft_create_data does (src/noncart/nufft.c:837,
 * 898): rolloff_correction() with a float beta calls kb_init()
 * (src/noncart/grid.c:45-60, 536-556), which fills the table by
 * kb_precompute() (src/noncart/grid.c:86-97) with bessel_i0()
 * (src/num/specfun.c:120-129).
 */
#include <complex.h>
#include <stdio.h>
#include <stdlib.h>

#include "num/init.h"
#include "noncart/grid.h"

int main(int argc, char* argv[])
{
	float os = (argc > 2) ? (float)atof(argv[1]) : 2.f;
	float width = (argc > 2) ? (float)atof(argv[2]) : 6.f;

	num_init();

	double beta = calc_beta(os, width);
	printf("beta %a\n", beta);

	// the roll-off of each requested axis length (a 1D image [n, 1, 1]);
	// the first call initialises the table with beta rounded to float
	int nroll = (argc > 3) ? (argc - 3) : 1;

	for (int a = 0; a < nroll; a++) {

		long n = (argc > 3) ? atol(argv[3 + a]) : 256;
		long dims[3] = { n, 1, 1 };
		complex float* roll = malloc(sizeof(complex float) * n);
		rolloff_correction(os, width, beta, dims, roll);

		for (long x = 0; x < n; x++)
			printf("roll %ld %ld %a\n", n, x, crealf(roll[x]));

		free(roll);
	}

	printf("i0beta %a\n", bessel_kb_beta);

	float* table = malloc(sizeof(float) * (kb_size + 1));
	kb_precompute((float)beta, kb_size, table);

	for (int i = 0; i <= kb_size; i++)
		printf("kb %d %a\n", i, table[i]);

	free(table);
	return 0;
}
