/*
 * Mufflon's header name for the core C ABI (src/core/export/core_interface.h),
 * so that code written against the reference, such as examples/example.c,
 * compiles unchanged. Everything is declared in mufflon_core.h.
 */
#ifndef MUFFLON_B200_CORE_INTERFACE_H
#define MUFFLON_B200_CORE_INTERFACE_H
#include "mufflon_core.h"
#endif
