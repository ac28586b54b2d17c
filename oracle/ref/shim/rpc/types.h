/* Sun RPC basic types for the XDR stand-in (CPU oracle build only). */
#ifndef HB_REF_SHIM_RPC_TYPES_H
#define HB_REF_SHIM_RPC_TYPES_H
typedef int bool_t;
typedef char* caddr_t;
typedef unsigned int u_int;
#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif
#endif
