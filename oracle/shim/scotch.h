/*
 * Declaration-only stand-in for the SCOTCH header that the reference includes
 * unconditionally (src/include/adh.h:19).  The reference's serial SW2 path uses
 * no SCOTCH function; the three files that do (src/structs/sgrid/sgrid_reorder.c,
 * sgrid_repartition.c, src/messg/scotch_part_kway.c) are left out of the oracle
 * build, so only the integer type name is needed here.
 *
 * Test infrastructure only.
 */
#ifndef ORACLE_SHIM_SCOTCH_H
#define ORACLE_SHIM_SCOTCH_H
typedef int SCOTCH_Num;
#endif
