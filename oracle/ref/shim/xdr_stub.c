/* XDR stand-in for building HemePure as the CPU oracle (test infrastructure only).
 * Big-endian four-byte units per RFC 4506; 16-bit integers take a full unit,
 * 64-bit integers and doubles two units (high word first). */
#include <stdlib.h>
#include <string.h>
#include "rpc/xdr.h"

void xdrmem_create(XDR* x, char* addr, unsigned size, enum xdr_op op) {
  x->x_op = op;
  x->buf = addr;
  x->size = size;
  x->pos = 0;
  x->file = NULL;
}
void xdrstdio_create(XDR* x, FILE* file, enum xdr_op op) {
  x->x_op = op;
  x->buf = NULL;
  x->size = 0;
  x->pos = 0;
  x->file = file;
}
void xdr_destroy(XDR* x) {
  if (x->file) fflush(x->file);
}
unsigned xdr_getpos(XDR* x) { return x->file ? (unsigned)ftell(x->file) : x->pos; }
bool_t xdr_setpos(XDR* x, unsigned pos) {
  if (x->file) return fseek(x->file, (long)pos, SEEK_SET) == 0;
  if (pos > x->size) return FALSE;
  x->pos = pos;
  return TRUE;
}

static bool_t put_bytes(XDR* x, const unsigned char* b, unsigned n) {
  if (x->file) return fwrite(b, 1, n, x->file) == n;
  if (x->pos + n > x->size) return FALSE;
  memcpy(x->buf + x->pos, b, n);
  x->pos += n;
  return TRUE;
}
static bool_t get_bytes(XDR* x, unsigned char* b, unsigned n) {
  if (x->file) return fread(b, 1, n, x->file) == n;
  if (x->pos + n > x->size) return FALSE;
  memcpy(b, x->buf + x->pos, n);
  x->pos += n;
  return TRUE;
}
static bool_t unit32(XDR* x, uint32_t* v) {
  unsigned char b[4];
  if (x->x_op == XDR_ENCODE) {
    b[0] = (unsigned char)(*v >> 24);
    b[1] = (unsigned char)(*v >> 16);
    b[2] = (unsigned char)(*v >> 8);
    b[3] = (unsigned char)(*v);
    return put_bytes(x, b, 4);
  }
  if (x->x_op == XDR_DECODE) {
    if (!get_bytes(x, b, 4)) return FALSE;
    *v = ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | (uint32_t)b[3];
    return TRUE;
  }
  return TRUE;
}
static bool_t unit64(XDR* x, uint64_t* v) {
  uint32_t hi = (uint32_t)(*v >> 32), lo = (uint32_t)*v;
  if (!unit32(x, &hi) || !unit32(x, &lo)) return FALSE;
  if (x->x_op == XDR_DECODE) *v = ((uint64_t)hi << 32) | lo;
  return TRUE;
}
bool_t xdr_u_int(XDR* x, unsigned* v) {
  uint32_t u = *v;
  if (!unit32(x, &u)) return FALSE;
  *v = u;
  return TRUE;
}
bool_t xdr_int(XDR* x, int* v) {
  uint32_t u = (uint32_t)*v;
  if (!unit32(x, &u)) return FALSE;
  *v = (int)u;
  return TRUE;
}
bool_t xdr_int32_t(XDR* x, int32_t* v) { return xdr_int(x, (int*)v); }
bool_t xdr_uint32_t(XDR* x, uint32_t* v) { return unit32(x, v); }
bool_t xdr_int16_t(XDR* x, int16_t* v) {
  uint32_t u = (uint32_t)(int32_t)*v;
  if (!unit32(x, &u)) return FALSE;
  *v = (int16_t)(int32_t)u;
  return TRUE;
}
bool_t xdr_uint16_t(XDR* x, uint16_t* v) {
  uint32_t u = *v;
  if (!unit32(x, &u)) return FALSE;
  *v = (uint16_t)u;
  return TRUE;
}
bool_t xdr_int64_t(XDR* x, int64_t* v) { return unit64(x, (uint64_t*)v); }
bool_t xdr_uint64_t(XDR* x, uint64_t* v) { return unit64(x, v); }
bool_t xdr_float(XDR* x, float* v) {
  uint32_t u;
  memcpy(&u, v, 4);
  if (!unit32(x, &u)) return FALSE;
  memcpy(v, &u, 4);
  return TRUE;
}
bool_t xdr_double(XDR* x, double* v) {
  uint64_t u;
  memcpy(&u, v, 8);
  if (!unit64(x, &u)) return FALSE;
  memcpy(v, &u, 8);
  return TRUE;
}
bool_t xdr_string(XDR* x, char** s, unsigned maxsize) {
  static const unsigned char zeros[4] = {0, 0, 0, 0};
  uint32_t n = 0;
  if (x->x_op == XDR_ENCODE) {
    n = (uint32_t)strlen(*s);
    if (n > maxsize) return FALSE;
    if (!unit32(x, &n) || !put_bytes(x, (const unsigned char*)*s, n)) return FALSE;
    return put_bytes(x, zeros, (4 - n % 4) % 4);
  }
  if (x->x_op == XDR_DECODE) {
    unsigned char pad[4];
    if (!unit32(x, &n) || n > maxsize) return FALSE;
    if (*s == NULL) {
      *s = (char*)malloc(n + 1);
      if (!*s) return FALSE;
    }
    if (!get_bytes(x, (unsigned char*)*s, n)) return FALSE;
    (*s)[n] = '\0';
    return get_bytes(x, pad, (4 - n % 4) % 4);
  }
  if (x->x_op == XDR_FREE && *s) {
    free(*s);
    *s = NULL;
  }
  return TRUE;
}
bool_t xdr_wrapstring(XDR* x, char** s) { return xdr_string(x, s, ~0u); }
