/*
 * msd_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity oracle).
 *
 * A plain-C restatement, written for this repository, of the reference's
 * stable MSD radix string sort msd_CE6 (rantala/string-sorting,
 * src/msd_ce.cpp:367-419) together with the LCP definition the GPU sort
 * emits (src/mergesort_lcp.cpp:88-100).  Only the test suite, the smoke
 * check and the CPU-baseline leg of the benchmark load this library; the
 * product path (libssort_b200.so) never links or calls it.
 *
 * Parity is pinned two ways: against golden vectors produced by running the
 * reference's own msd_CE6 (committed under tests/golden/), and against the
 * reference library compiled from its sources into oracle/_ref/ when present.
 *
 * Differences from the reference that do not change the output:
 *   - the sort permutes an array of string indices (v[i]) instead of the
 *     pointer array itself; the string of index j is ptrs[j].  The reference
 *     sorts pointers; stable sorting of indices gives the same order.
 *   - recursion is replaced by an explicit work stack so that very long
 *     shared prefixes cannot overflow the C stack.  Buckets are disjoint, so
 *     the order in which they are refined does not change the result.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
	size_t start;
	size_t n;
	size_t depth;
} work_item;

typedef struct {
	work_item *items;
	size_t len, cap;
} work_stack;

static int push(work_stack *st, size_t start, size_t n, size_t depth)
{
	if (st->len == st->cap) {
		size_t nc = st->cap ? st->cap * 2 : 1024;
		work_item *p = (work_item *)realloc(st->items, nc * sizeof(work_item));
		if (!p)
			return -1;
		st->items = p;
		st->cap = nc;
	}
	st->items[st->len].start = start;
	st->items[st->len].n = n;
	st->items[st->len].depth = depth;
	st->len++;
	return 0;
}

/* get_char<uint16_t> (src/util/get_char.h:42-50): big-endian pair of bytes,
 * zero after the terminating NUL. */
static inline uint16_t superchar(const unsigned char *s, size_t depth)
{
	uint16_t c = s[depth];
	if (c)
		c = (uint16_t)((c << 8) | s[depth + 1]);
	return c;
}

/* insertion_sort (src/util/insertion_sort.h:29-48): stable, compares from
 * `depth` until the first difference or the end of the left string. */
static void insertion(const unsigned char *const *ptrs, uint32_t *v, size_t n,
		      size_t depth)
{
	for (size_t i = 1; i < n; ++i) {
		uint32_t cur = v[i];
		const unsigned char *t0 = ptrs[cur] + depth;
		size_t j = i;
		while (j > 0) {
			const unsigned char *s = ptrs[v[j - 1]] + depth;
			const unsigned char *t = t0;
			while (*s == *t && *s != 0) {
				++s;
				++t;
			}
			if (*s <= *t)
				break;
			v[j] = v[j - 1];
			--j;
		}
		v[j] = cur;
	}
}

/*
 * The sort proper.  Segments with n >= 0x10000 take one 16-bit-superalphabet
 * counting-sort step (src/msd_ce.cpp:367-407); smaller ones take 8-bit
 * steps (msd_CE2_16bit_5, src/msd_ce.cpp:293-320); n < 32 goes to insertion
 * sort.  A bucket whose (low) character is NUL holds only finished strings
 * and is not refined further (src/msd_ce.cpp:306-307 and :402).
 */
static int msd_sort_indices(const unsigned char *const *ptrs, uint32_t *v,
			    size_t n)
{
	if (n < 2)
		return 0;
	uint16_t *dig = (uint16_t *)malloc(n * sizeof(uint16_t));
	uint32_t *tmp = (uint32_t *)malloc(n * sizeof(uint32_t));
	size_t *cnt16 = (size_t *)malloc(0x10000 * sizeof(size_t));
	work_stack st = {0, 0, 0};
	int rc = 0;
	if (!dig || !tmp || !cnt16 || push(&st, 0, n, 0)) {
		rc = -1;
		goto out;
	}
	while (st.len) {
		work_item w = st.items[--st.len];
		uint32_t *a = v + w.start;
		size_t m = w.n;
		size_t depth = w.depth;
		if (m < 32) {
			insertion(ptrs, a, m, depth);
			continue;
		}
		if (m >= 0x10000) {
			memset(cnt16, 0, 0x10000 * sizeof(size_t));
			for (size_t i = 0; i < m; ++i) {
				dig[i] = superchar(ptrs[a[i]], depth);
				cnt16[dig[i]]++;
			}
			size_t sum = 0;
			for (size_t c = 0; c < 0x10000; ++c) {
				size_t k = cnt16[c];
				cnt16[c] = sum;
				sum += k;
			}
			for (size_t i = 0; i < m; ++i)
				tmp[cnt16[dig[i]]++] = a[i];
			memcpy(a, tmp, m * sizeof(uint32_t));
			/* cnt16[c] now holds the end of bucket c. */
			size_t begin = 0;
			for (size_t c = 0; c < 0x10000; ++c) {
				size_t end = cnt16[c];
				size_t k = end - begin;
				if (k > 1 && (c & 0xFF)) {
					if (push(&st, w.start + begin, k, depth + 2)) {
						rc = -1;
						goto out;
					}
				}
				begin = end;
			}
		} else {
			size_t cnt[256];
			memset(cnt, 0, sizeof(cnt));
			unsigned char *d8 = (unsigned char *)dig;
			for (size_t i = 0; i < m; ++i) {
				d8[i] = ptrs[a[i]][depth];
				cnt[d8[i]]++;
			}
			size_t sum = 0;
			for (int c = 0; c < 256; ++c) {
				size_t k = cnt[c];
				cnt[c] = sum;
				sum += k;
			}
			for (size_t i = 0; i < m; ++i)
				tmp[cnt[d8[i]]++] = a[i];
			memcpy(a, tmp, m * sizeof(uint32_t));
			size_t begin = cnt[0];
			for (int c = 1; c < 256; ++c) {
				size_t end = cnt[c];
				size_t k = end - begin;
				if (k > 1) {
					if (push(&st, w.start + begin, k, depth + 1)) {
						rc = -1;
						goto out;
					}
				}
				begin = end;
			}
		}
	}
out:
	free(st.items);
	free(dig);
	free(tmp);
	free(cnt16);
	return rc;
}

/* lcp() (src/mergesort_lcp.cpp:88-100): equal leading bytes, stopping at the
 * first difference or at the NUL of the left string. */
static uint32_t lcp_pair(const unsigned char *a, const unsigned char *b)
{
	uint32_t i = 0;
	while (a[i] != 0 && a[i] == b[i])
		++i;
	return i;
}

/*
 * Sort the strings ptrs[0..n) (each NUL-terminated).  perm_out[i] receives
 * the index of the string at sorted position i; lcp_out (optional) receives
 * lcp_out[0] = 0 and lcp_out[i] = lcp(s[perm[i-1]], s[perm[i]]).
 * Returns 0, or -1 when memory runs out.
 */
int oracle_sort_ptrs(const unsigned char *const *ptrs, size_t n,
		     uint32_t *perm_out, uint32_t *lcp_out)
{
	for (size_t i = 0; i < n; ++i)
		perm_out[i] = (uint32_t)i;
	if (msd_sort_indices(ptrs, perm_out, n))
		return -1;
	if (lcp_out && n) {
		lcp_out[0] = 0;
		for (size_t i = 1; i < n; ++i)
			lcp_out[i] = lcp_pair(ptrs[perm_out[i - 1]], ptrs[perm_out[i]]);
	}
	return 0;
}

/* The same over an arena: string i starts at arena + offs[i]; offs holds
 * 32-bit (off_width 4) or 64-bit (off_width 8) unsigned offsets. */
int oracle_sort_arena(const unsigned char *arena, const void *offs, int off_width,
		      size_t n, uint32_t *perm_out, uint32_t *lcp_out)
{
	if (off_width != 4 && off_width != 8)
		return -2;
	const unsigned char **ptrs =
		(const unsigned char **)malloc((n ? n : 1) * sizeof(*ptrs));
	if (!ptrs)
		return -1;
	for (size_t i = 0; i < n; ++i) {
		uint64_t o = off_width == 4 ? ((const uint32_t *)offs)[i]
					    : ((const uint64_t *)offs)[i];
		ptrs[i] = arena + o;
	}
	int rc = oracle_sort_ptrs(ptrs, n, perm_out, lcp_out);
	free(ptrs);
	return rc;
}

/* In-place pointer-array form with the routine signature
 * void(unsigned char**, size_t) (src/routine.h:33). */
void oracle_msd(unsigned char **strings, size_t n)
{
	if (n < 2)
		return;
	uint32_t *perm = (uint32_t *)malloc(n * sizeof(uint32_t));
	unsigned char **orig = (unsigned char **)malloc(n * sizeof(*orig));
	if (!perm || !orig)
		abort();
	memcpy(orig, strings, n * sizeof(*orig));
	if (oracle_sort_ptrs((const unsigned char *const *)orig, n, perm, NULL))
		abort();
	for (size_t i = 0; i < n; ++i)
		strings[i] = orig[perm[i]];
	free(perm);
	free(orig);
}

/*
 * Independent checker: verifies that perm is a permutation of [0,n), that
 * adjacent strings are in byte order, that equal strings keep ascending index
 * (stability), and, when lcp is given, every lcp entry.  Returns the number of
 * violations found (0 = valid); *first_bad receives the first bad position.
 */
size_t oracle_check(const unsigned char *const *ptrs, size_t n,
		    const uint32_t *perm, const uint32_t *lcp, size_t *first_bad)
{
	size_t bad = 0;
	size_t fb = (size_t)-1;
	unsigned char *seen = (unsigned char *)calloc(n ? n : 1, 1);
	if (!seen)
		return (size_t)-1;
	for (size_t i = 0; i < n; ++i) {
		uint32_t p = perm[i];
		if (p >= n || seen[p]) {
			++bad;
			if (fb == (size_t)-1)
				fb = i;
			continue;
		}
		seen[p] = 1;
	}
	free(seen);
	if (bad)
		goto done;
	if (lcp && n && lcp[0] != 0) {
		++bad;
		fb = 0;
	}
	for (size_t i = 1; i < n; ++i) {
		const unsigned char *a = ptrs[perm[i - 1]];
		const unsigned char *b = ptrs[perm[i]];
		uint32_t l = lcp_pair(a, b);
		int c = (int)a[l] - (int)b[l];
		int ok = c < 0 || (c == 0 && perm[i - 1] < perm[i]);
		if (lcp && lcp[i] != l)
			ok = 0;
		if (!ok) {
			++bad;
			if (fb == (size_t)-1)
				fb = i;
		}
	}
done:
	if (first_bad)
		*first_bad = fb;
	return bad;
}

size_t oracle_check_arena(const unsigned char *arena, const void *offs,
			  int off_width, size_t n, const uint32_t *perm,
			  const uint32_t *lcp, size_t *first_bad)
{
	const unsigned char **ptrs =
		(const unsigned char **)malloc((n ? n : 1) * sizeof(*ptrs));
	if (!ptrs)
		return (size_t)-1;
	for (size_t i = 0; i < n; ++i) {
		uint64_t o = off_width == 4 ? ((const uint32_t *)offs)[i]
					    : ((const uint64_t *)offs)[i];
		ptrs[i] = arena + o;
	}
	size_t r = oracle_check(ptrs, n, perm, lcp, first_bad);
	free(ptrs);
	return r;
}
