/*
 * Link stubs for symbols that the reference sources reference but define
 * nowhere in the vendored tree (they live in the un-vendored companion
 * library or in Pardiso).  None is on the CPR-GMRES path; each aborts if it
 * is ever reached, so a silent wrong answer is impossible.
 */
#include <stdio.h>
#include <stdlib.h>

#define JXCPR_REF_STUB(name)                                                   \
    void name(void)                                                            \
    {                                                                          \
        fprintf(stderr, "oracle: unavailable reference symbol %s\n", #name);   \
        abort();                                                               \
    }

JXCPR_REF_STUB(jxf_BigBinarySearch)
JXCPR_REF_STUB(jxf_BigQsort0)
JXCPR_REF_STUB(jxf_BoomerAMGBuildCoarseOperator)
JXCPR_REF_STUB(jxf_CSRMatrixExtractDiagonal)
JXCPR_REF_STUB(jxf_ParCSRCommPkgGetRemoteData_Complex)
JXCPR_REF_STUB(jxf_ParCSRCommPkgGetRemoteData_Int)
JXCPR_REF_STUB(jxf_ParCSRCommPkgGetRemoteRankArray)
JXCPR_REF_STUB(jxf_ParCSRMatrixClone)
JXCPR_REF_STUB(jxf_ParCSRMatrixReorder)
JXCPR_REF_STUB(jxf_ParMatmul_NozeroStruct)
JXCPR_REF_STUB(jxf_pardiso)
