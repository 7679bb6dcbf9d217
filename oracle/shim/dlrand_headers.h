/* Oracle shim (test infrastructure): dlrand_headers.h is instantiated by the
 * reference headers but nothing on the SpMV/CG path uses it. */
