/* XDR (RFC 4506) encoding and decoding over a memory buffer or a stdio stream,
 * covering the calls HemePure's io/writers/xdr classes make (CPU oracle build
 * only).  Every item occupies a multiple of four big-endian bytes. */
#ifndef HB_REF_SHIM_RPC_XDR_H
#define HB_REF_SHIM_RPC_XDR_H
#include <stdint.h>
#include <stdio.h>
#include "rpc/types.h"
#ifdef __cplusplus
extern "C" {
#endif
enum xdr_op { XDR_ENCODE = 0, XDR_DECODE = 1, XDR_FREE = 2 };
typedef struct XDR {
  enum xdr_op x_op;
  char* buf;       /* memory stream, or NULL for stdio */
  unsigned size;
  unsigned pos;
  FILE* file;      /* stdio stream, or NULL for memory */
} XDR;
void xdrmem_create(XDR* x, char* addr, unsigned size, enum xdr_op op);
void xdrstdio_create(XDR* x, FILE* file, enum xdr_op op);
void xdr_destroy(XDR* x);
unsigned xdr_getpos(XDR* x);
bool_t xdr_setpos(XDR* x, unsigned pos);
bool_t xdr_int(XDR* x, int* v);
bool_t xdr_u_int(XDR* x, unsigned* v);
bool_t xdr_int16_t(XDR* x, int16_t* v);
bool_t xdr_uint16_t(XDR* x, uint16_t* v);
bool_t xdr_int32_t(XDR* x, int32_t* v);
bool_t xdr_uint32_t(XDR* x, uint32_t* v);
bool_t xdr_int64_t(XDR* x, int64_t* v);
bool_t xdr_uint64_t(XDR* x, uint64_t* v);
bool_t xdr_float(XDR* x, float* v);
bool_t xdr_double(XDR* x, double* v);
bool_t xdr_string(XDR* x, char** s, unsigned maxsize);
bool_t xdr_wrapstring(XDR* x, char** s);
#ifdef __cplusplus
}
#endif
#endif
