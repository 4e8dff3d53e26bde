/* fdtd_oracle.c — TEST INFRASTRUCTURE ONLY: the CPU oracle for the CUDA engine.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * the library built from this file, and only as the checker.  The engine
 * never links, loads or calls it.
 *
 * Two instantiations of the same restatement (fdtd_oracle_body.h):
 *   orc_*    float  — bit-exact with the reference's acoustic_fdtd.cpp when
 *                     both are compiled with -ffp-contract=off;
 *   orc64_*  double — FP64 oracle for the storage-precision study.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off -fPIC -shared).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#include <math.h>

#define EXPORT __attribute__((visibility("default")))

/* float instantiation */
#define R float
#define L(x) x##f
#define P_(name) orc_##name
#define S_ OrcState32
#include "fdtd_oracle_body.h"
#undef R
#undef L
#undef P_
#undef S_

/* double instantiation */
#define R double
#define L(x) x
#define P_(name) orc64_##name
#define S_ OrcState64
#include "fdtd_oracle_body.h"
#undef R
#undef L
#undef P_
#undef S_
