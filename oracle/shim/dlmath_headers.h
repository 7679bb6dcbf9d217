/* X-macro: the one math helper the hot-path files use (exclusive prefix sum
 * in place, the shifted-by-one CSR build of src/matrix.c:411-437).
 * Oracle shim (test infrastructure), project-written. */
static inline void DLSHIM_CAT(DLMATH_PREFIX, prefixsum_exc)(
    DLMATH_TYPE_T * a, size_t n)
{
  size_t i;
  DLMATH_TYPE_T run = 0, t;
  for (i = 0; i < n; ++i) {
    t = a[i];
    a[i] = run;
    run += t;
  }
}
