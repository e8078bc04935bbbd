/* Minimal stand-in for the SUNDIALS type header, written for this checker:
 * just the scalar types and macros the reference's 2d_i2 sources use, so
 * those sources compile without a SUNDIALS installation.  TEST
 * INFRASTRUCTURE ONLY (oracle/ref_i2). */
#ifndef LLG_SHIM_SUNDIALS_TYPES_H
#define LLG_SHIM_SUNDIALS_TYPES_H
typedef double sunrealtype;
typedef int sunbooleantype;
typedef long sunindextype;
typedef int SUNErrCode;
#define SUN_RCONST(x) (x)
#define SUNTRUE 1
#define SUNFALSE 0
typedef struct llg_shim_context* SUNContext;
#define SUN_COMM_NULL 0
#ifdef __cplusplus
extern "C" {
#endif
int SUNContext_Create(int comm, SUNContext* ctx);
int SUNContext_Free(SUNContext* ctx);
#ifdef __cplusplus
}
#endif
#endif
