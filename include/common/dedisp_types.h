/*
 * dedisp_types.h -- scalar types and flags of the dedisp interface.
 * Same definitions and include guard as the reference
 * src/common/dedisp_types.h:6-36, so either copy may be included first.
 */
#ifndef DEDISP_TYPES_H_INCLUDE_GUARD
#define DEDISP_TYPES_H_INCLUDE_GUARD
typedef float         dedisp_float;
typedef unsigned char dedisp_byte;
typedef unsigned long dedisp_size;
typedef int           dedisp_bool;
typedef unsigned int  dedisp_word;
typedef struct { float real; float imag; } dedisp_float2;

/* Flags: src/common/dedisp_types.h:29-36 */
typedef enum {
    DEDISP_USE_DEFAULT     = 0,
    DEDISP_HOST_POINTERS   = 1 << 1,
    DEDISP_DEVICE_POINTERS = 1 << 2,
    DEDISP_WAIT            = 1 << 3,
    DEDISP_ASYNC           = 1 << 4
} dedisp_flag;
#endif /* DEDISP_TYPES_H_INCLUDE_GUARD */
