/* seeded_rand.h -- forced into the reference's Maslov sources by
 * oracle/Makefile (g++ -include).  The reference draws its swap attempts from
 * the C runtime's rand(), 15 bits per call on the Microsoft runtime it was
 * built with (hence its (rand() * 0x8000 + rand()) % M), seeded by
 * srand(time(0)).  Here rand() is that 15-bit linear congruential generator
 * (state = state * 214013 + 2531011, output = bits 16..30 of the state), and
 * srand() ignores its argument and seeds from ref_rand_seed, which the test
 * driver sets before each call, so runs are reproducible. */
#include <stdlib.h>
#include <time.h>
#ifdef __cplusplus
extern "C" {
#endif
extern unsigned int ref_rand_seed;
int ref_rand15(void);
void ref_srand15(unsigned int seed);
#ifdef __cplusplus
}
#endif
#define rand() ref_rand15()
#define srand(x) ref_srand15(ref_rand_seed)
