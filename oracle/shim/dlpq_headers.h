/* X-macro: indexed binary-heap priority queue for DLPQ_PREFIX / DLPQ_KEY_T /
 * DLPQ_VAL_T, with DLPQ_MIN selecting a min-queue and DLPQ_STATIC making the
 * functions file-local.
 *
 * Oracle shim (test infrastructure), project-written from the call sites in
 * the reference's src/permute.c:26-36,60-109: create(start,end) over values in
 * [start,end), push(key,val), pop() -> val, contains(val), remove(val),
 * free(), and a public `size` field.  It is not domlib's dlpq.
 *
 * Ordering: entries compare by key, and entries with equal keys by value
 * (smaller value first for a min-queue).  That makes the pop order a pure
 * function of the (key, value) pairs present, so a restatement that orders
 * ties the same way reproduces permute.c's results exactly.  domlib's own
 * tie order is not known (the submodule is not vendored).
 *
 * No include guard on purpose: instantiated once per prefix. */
#include <stdlib.h>

#ifndef DLPQ_MIN
#define DLPQ_MIN 0
#endif

#ifdef DLPQ_STATIC
#define DLPQ_SHIM_FN static inline
#else
#define DLPQ_SHIM_FN inline
#endif

#define DLPQ_SHIM_T DLSHIM_CAT(DLPQ_PREFIX, pq_t)
#define DLPQ_SHIM_NAME(name) DLSHIM_CAT(DLSHIM_CAT(DLPQ_PREFIX, pq), name)

typedef struct {
  DLPQ_KEY_T key;
  DLPQ_VAL_T val;
} DLSHIM_CAT(DLPQ_PREFIX, pq_entry_t);

typedef struct {
  size_t size;
  DLPQ_VAL_T start;
  DLPQ_VAL_T end;
  DLSHIM_CAT(DLPQ_PREFIX, pq_entry_t) * heap; /* [end-start] entries        */
  size_t * where;                             /* heap slot of val, or (size_t)-1 */
} DLPQ_SHIM_T;

/* a before b in pop order */
DLPQ_SHIM_FN int DLPQ_SHIM_NAME(before_)(DLPQ_KEY_T ka, DLPQ_VAL_T va,
    DLPQ_KEY_T kb, DLPQ_VAL_T vb)
{
#if DLPQ_MIN
  return ka < kb || (ka == kb && va < vb);
#else
  return ka > kb || (ka == kb && va < vb);
#endif
}

DLPQ_SHIM_FN void DLPQ_SHIM_NAME(place_)(DLPQ_SHIM_T * q, size_t slot,
    DLSHIM_CAT(DLPQ_PREFIX, pq_entry_t) e)
{
  q->heap[slot] = e;
  q->where[e.val - q->start] = slot;
}

DLPQ_SHIM_FN void DLPQ_SHIM_NAME(up_)(DLPQ_SHIM_T * q, size_t slot)
{
  DLSHIM_CAT(DLPQ_PREFIX, pq_entry_t) const e = q->heap[slot];
  while (slot > 0) {
    size_t const parent = (slot - 1) / 2;
    if (!DLPQ_SHIM_NAME(before_)(e.key, e.val, q->heap[parent].key,
          q->heap[parent].val)) {
      break;
    }
    DLPQ_SHIM_NAME(place_)(q, slot, q->heap[parent]);
    slot = parent;
  }
  DLPQ_SHIM_NAME(place_)(q, slot, e);
}

DLPQ_SHIM_FN void DLPQ_SHIM_NAME(down_)(DLPQ_SHIM_T * q, size_t slot)
{
  DLSHIM_CAT(DLPQ_PREFIX, pq_entry_t) const e = q->heap[slot];
  for (;;) {
    size_t best = slot;
    DLPQ_KEY_T bk = e.key;
    DLPQ_VAL_T bv = e.val;
    size_t c;
    for (c = 2 * slot + 1; c <= 2 * slot + 2 && c < q->size; ++c) {
      if (DLPQ_SHIM_NAME(before_)(q->heap[c].key, q->heap[c].val, bk, bv)) {
        best = c;
        bk = q->heap[c].key;
        bv = q->heap[c].val;
      }
    }
    if (best == slot) {
      break;
    }
    DLPQ_SHIM_NAME(place_)(q, slot, q->heap[best]);
    slot = best;
  }
  DLPQ_SHIM_NAME(place_)(q, slot, e);
}

DLPQ_SHIM_FN DLPQ_SHIM_T * DLPQ_SHIM_NAME(create)(DLPQ_VAL_T start, DLPQ_VAL_T end)
{
  size_t const n = end > start ? (size_t)(end - start) : 0;
  size_t i;
  DLPQ_SHIM_T * q = (DLPQ_SHIM_T *)malloc(sizeof(DLPQ_SHIM_T));
  q->size = 0;
  q->start = start;
  q->end = end;
  q->heap = malloc((n ? n : 1) * sizeof(*q->heap));
  q->where = (size_t *)malloc((n ? n : 1) * sizeof(size_t));
  for (i = 0; i < n; ++i) {
    q->where[i] = (size_t)-1;
  }
  return q;
}

DLPQ_SHIM_FN void DLPQ_SHIM_NAME(push)(DLPQ_KEY_T key, DLPQ_VAL_T val, DLPQ_SHIM_T * q)
{
  DLSHIM_CAT(DLPQ_PREFIX, pq_entry_t) e;
  e.key = key;
  e.val = val;
  q->heap[q->size] = e;
  q->where[val - q->start] = q->size;
  ++q->size;
  DLPQ_SHIM_NAME(up_)(q, q->size - 1);
}

DLPQ_SHIM_FN int DLPQ_SHIM_NAME(contains)(DLPQ_VAL_T val, DLPQ_SHIM_T const * q)
{
  return q->where[val - q->start] != (size_t)-1;
}

DLPQ_SHIM_FN void DLPQ_SHIM_NAME(remove)(DLPQ_VAL_T val, DLPQ_SHIM_T * q)
{
  size_t const slot = q->where[val - q->start];
  size_t const last = q->size - 1;
  q->where[val - q->start] = (size_t)-1;
  --q->size;
  if (slot != last) {
    DLPQ_SHIM_NAME(place_)(q, slot, q->heap[last]);
    /* the moved entry goes up or down; if it went up, the entry now in
     * `slot` came from above and down_ leaves it there */
    DLPQ_SHIM_NAME(up_)(q, slot);
    DLPQ_SHIM_NAME(down_)(q, slot);
  }
}

DLPQ_SHIM_FN DLPQ_VAL_T DLPQ_SHIM_NAME(pop)(DLPQ_SHIM_T * q)
{
  DLPQ_VAL_T const top = q->heap[0].val;
  DLPQ_SHIM_NAME(remove)(top, q);
  return top;
}

DLPQ_SHIM_FN void DLPQ_SHIM_NAME(free)(DLPQ_SHIM_T * q)
{
  free(q->heap);
  free(q->where);
  free(q);
}

#undef DLPQ_SHIM_NAME
#undef DLPQ_SHIM_T
#undef DLPQ_SHIM_FN
