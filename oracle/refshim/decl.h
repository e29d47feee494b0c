/* Force-included into every reference source file when the reference CPU library is
 * compiled as an oracle (see oracle/Makefile).  The reference sources rely on headers
 * that older toolchains pulled in transitively, and on the C symbols Fr_raw* / Fq_raw*
 * that normally come from NASM-generated assembly (fr.casm, fq.casm) which cannot be
 * assembled here.  Declaring them extern "C" here gives ff.cpp's own Fr_toMont /
 * Fr_fromMont definitions C linkage, matching fr.h / fq.h. */
#ifndef CUSNARKS_B200_REFSHIM_DECL_H
#define CUSNARKS_B200_REFSHIM_DECL_H
#include <cstring>
#include <cstdint>
#include <algorithm>
#include <pthread.h>
#include <sys/sysinfo.h>
extern "C" {
void Fr_rawAdd(uint32_t *r, const uint32_t *a, const uint32_t *b);
void Fr_rawSub(uint32_t *r, const uint32_t *a, const uint32_t *b);
void Fr_rawMMul(uint32_t *r, const uint32_t *a, const uint32_t *b);
void Fr_rawMSquare(uint32_t *r, const uint32_t *a);
void Fr_toMont(uint32_t *z, const uint32_t *x);
void Fr_fromMont(uint32_t *z, const uint32_t *x);
void Fq_rawAdd(uint32_t *r, const uint32_t *a, const uint32_t *b);
void Fq_rawSub(uint32_t *r, const uint32_t *a, const uint32_t *b);
void Fq_rawMMul(uint32_t *r, const uint32_t *a, const uint32_t *b);
void Fq_rawMSquare(uint32_t *r, const uint32_t *a);
void Fq_toMont(uint32_t *z, const uint32_t *x);
void Fq_fromMont(uint32_t *z, const uint32_t *x);
}
#endif
