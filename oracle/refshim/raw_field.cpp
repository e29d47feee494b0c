/* C definitions of the Fr_raw* / Fq_raw* symbols that the reference's ff.cpp hands out
 * through getcb_{addm,subm,mulm,sqm}_h.  In the reference they are NASM assembly
 * (fr.casm = modulus q, MOD_GROUP; fq.casm = modulus r, MOD_FIELD).  Here they forward to
 * the reference's own portable C routines (montmult_h FIOS, addm_h, subm_h) with the
 * matching modulus index.  Montgomery products reduced to [0,p) are unique, so the
 * results are the same words the assembly would return.  Oracle build only. */
#include <cstdint>
#include "types.h"
#include "ff.h"

extern "C" {
void Fr_rawAdd(uint32_t *r, const uint32_t *a, const uint32_t *b) { addm_h(r, a, b, 0); }
void Fr_rawSub(uint32_t *r, const uint32_t *a, const uint32_t *b) { subm_h(r, a, b, 0); }
void Fr_rawMMul(uint32_t *r, const uint32_t *a, const uint32_t *b) { montmult_h(r, a, b, 0); }
void Fr_rawMSquare(uint32_t *r, const uint32_t *a) { montmult_h(r, a, a, 0); }
void Fq_rawAdd(uint32_t *r, const uint32_t *a, const uint32_t *b) { addm_h(r, a, b, 1); }
void Fq_rawSub(uint32_t *r, const uint32_t *a, const uint32_t *b) { subm_h(r, a, b, 1); }
void Fq_rawMMul(uint32_t *r, const uint32_t *a, const uint32_t *b) { montmult_h(r, a, b, 1); }
void Fq_rawMSquare(uint32_t *r, const uint32_t *a) { montmult_h(r, a, a, 1); }
}
