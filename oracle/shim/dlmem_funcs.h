/* Oracle shim (test infrastructure): dlmem_funcs.h is instantiated by the
 * reference headers but nothing on the SpMV/CG path uses it. */
