/*
 * ref_shim.cpp -- TEST INFRASTRUCTURE ONLY.
 *
 * Compiled together with the reference's own sources (rantala/string-sorting:
 * src/msd_ce.cpp, src/multikey_cache.cpp, src/burstsort.cpp, src/routines.c,
 * external/parallel_string_radix_sort.cpp) into oracle/_ref/libref.so by
 * oracle/Makefile.  It exposes the reference routine registry through a plain
 * C entry point so the tests and the CPU-baseline leg of the benchmark can run
 * the unmodified reference routines (msd_CE6 as the oracle, msd_CE2 as the
 * cross-check, multikey_cache8 / burstsort_vector as extra baselines).
 *
 * Lookup follows routine_from_name (src/routines.c:43-51); the call is the
 * routine's own f(strings, n) (src/routine.h:32-37).
 */
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <chrono>
#include "routines.h"

extern "C" {

/* Run the registered reference routine `name` on strings[0..n).  Returns 0,
 * or -1 if no routine of that name is registered. */
int ref_sort(const char *name, unsigned char **strings, size_t n)
{
	const struct routine *r = routine_from_name(name);
	if (!r)
		return -1;
	if (n == 0)
		return 0;
	r->f(strings, n);
	return 0;
}

/* 1 if the routine is marked multicore, 0 if single core, -1 if unknown. */
int ref_is_multicore(const char *name)
{
	const struct routine *r = routine_from_name(name);
	if (!r)
		return -1;
	return r->multicore ? 1 : 0;
}

/* Seconds taken by routine `name` on the strings arena + offs[0..n): the
 * pointer array is built first and only the r->f(strings, n) call is timed
 * (steady clock; the reference's own timer truncates to whole milliseconds,
 * src/util/timing.c:52-53).  Returns -1 if the routine is unknown. */
double ref_time_sort(const char *name, const unsigned char *arena, const uint64_t *offs,
		     size_t n)
{
	const struct routine *r = routine_from_name(name);
	if (!r)
		return -1.0;
	unsigned char **s = (unsigned char **)malloc((n ? n : 1) * sizeof(*s));
	if (!s)
		return -2.0;
	for (size_t i = 0; i < n; ++i)
		s[i] = (unsigned char *)arena + offs[i];
	auto t0 = std::chrono::steady_clock::now();
	if (n)
		r->f(s, n);
	auto t1 = std::chrono::steady_clock::now();
	free(s);
	return std::chrono::duration<double>(t1 - t0).count();
}

/* Sort an arena (string i at arena + offs[i]) with routine `name` and write
 * the index permutation: perm[k] = original index of the k-th smallest.
 * Duplicate offsets are allowed only if the routine is stable and pointer
 * identity is not needed; the mapping back uses each pointer's position in a
 * copy sorted by address, so every offs[i] must be distinct. */
int ref_sort_arena_perm(const char *name, const unsigned char *arena,
			const uint64_t *offs, size_t n, uint32_t *perm)
{
	const struct routine *r = routine_from_name(name);
	if (!r)
		return -1;
	if (n == 0)
		return 0;
	unsigned char **s = (unsigned char **)malloc(n * sizeof(*s));
	if (!s)
		return -2;
	for (size_t i = 0; i < n; ++i)
		s[i] = (unsigned char *)arena + offs[i];
	r->f(s, n);
	/* offsets are distinct and ascending in the generators' arenas; recover
	 * indices by binary search over offs when ascending, else fail. */
	for (size_t i = 1; i < n; ++i) {
		if (offs[i] <= offs[i - 1]) {
			free(s);
			return -3;
		}
	}
	for (size_t k = 0; k < n; ++k) {
		uint64_t o = (uint64_t)(s[k] - arena);
		size_t lo = 0, hi = n;
		while (lo < hi) {
			size_t mid = lo + (hi - lo) / 2;
			if (offs[mid] < o)
				lo = mid + 1;
			else
				hi = mid;
		}
		perm[k] = (uint32_t)lo;
	}
	free(s);
	return 0;
}

}
