/*
 * Memory-allocator (MA) stand-in: the reference only calls MA_init once at
 * start-up (pjayci.c:38).  Test infrastructure only.
 */
#ifndef ORACLE_SHIM_MACDECLS_H
#define ORACLE_SHIM_MACDECLS_H

int MA_init(int type, long stack, long heap);

#endif
