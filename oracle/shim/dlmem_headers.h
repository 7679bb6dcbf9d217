/* X-macro: typed memory helpers for DLMEM_PREFIX / DLMEM_TYPE_T.
 * Oracle shim (test infrastructure), project-written; no include guard on
 * purpose because it is instantiated once per element type. */
static inline DLMEM_TYPE_T * DLSHIM_CAT(DLMEM_PREFIX, alloc)(size_t n)
{
  return (DLMEM_TYPE_T *)malloc((n ? n : 1) * sizeof(DLMEM_TYPE_T));
}
static inline DLMEM_TYPE_T * DLSHIM_CAT(DLMEM_PREFIX, calloc)(size_t n)
{
  return (DLMEM_TYPE_T *)calloc(n ? n : 1, sizeof(DLMEM_TYPE_T));
}
static inline DLMEM_TYPE_T * DLSHIM_CAT(DLMEM_PREFIX, set)(
    DLMEM_TYPE_T * dst, DLMEM_TYPE_T v, size_t n)
{
  size_t i;
  for (i = 0; i < n; ++i) {
    dst[i] = v;
  }
  return dst;
}
static inline DLMEM_TYPE_T * DLSHIM_CAT(DLMEM_PREFIX, copy)(
    DLMEM_TYPE_T * dst, DLMEM_TYPE_T const * src, size_t n)
{
  if (n) {
    memmove(dst, src, n * sizeof(DLMEM_TYPE_T));
  }
  return dst;
}
static inline DLMEM_TYPE_T * DLSHIM_CAT(DLMEM_PREFIX, init_alloc)(
    DLMEM_TYPE_T v, size_t n)
{
  return DLSHIM_CAT(DLMEM_PREFIX, set)(DLSHIM_CAT(DLMEM_PREFIX, alloc)(n), v, n);
}
