/* Stand-in: Gram-Schmidt and preconditioning-side selectors.  TEST
 * INFRASTRUCTURE ONLY. */
#ifndef LLG_SHIM_SUNDIALS_ITERATIVE_H
#define LLG_SHIM_SUNDIALS_ITERATIVE_H
#define SUN_PREC_NONE 0
#define SUN_PREC_LEFT 1
#define SUN_MODIFIED_GS 1
#define SUN_CLASSICAL_GS 2
#endif
