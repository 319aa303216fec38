/* lanczos_knobs.h -- harness-only Lanczos settings of the reference build.
 *
 * The reference hard-codes its Lanczos length and stop test as local constants:
 * mlanc = 40 (src/dmrg_inst.cpp:267) and |<v|Hv>|/|Hv| within 1e-8 of 1
 * (src/dmrg_inst.cpp:1338).  oracle/Makefile compiles a copy of that file in
 * which the two constants read these globals; ref_harness.cpp defines them with
 * the reference's values as defaults and sets them from -mlanc / -lanc_check. */
#pragma once
extern int ref_lanczos_mlanc;
extern double ref_lanczos_check;
