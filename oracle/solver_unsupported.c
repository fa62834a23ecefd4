/*
 * oracle/solver_unsupported.c -- entry points of src/solver that the
 * reference's C physics driver references but that lie outside the 2D
 * structured hot path (3D hanging faces and operators, unstructured faces).
 *
 * TEST INFRASTRUCTURE. They exist only so that src/physics/src/*.c links;
 * reaching one is a harness error, reported and ended.
 */
#include <stdio.h>
#include <stdlib.h>

#define UNSUPPORTED(name)                                                        \
    void name(void)                                                              \
    {                                                                            \
        fprintf(stderr, "oracle: %s is outside the 2D structured path\n", #name); \
        abort();                                                                 \
    }

UNSUPPORTED(solver_residual_face_full_hang_structured_3d)
UNSUPPORTED(solver_residual_face_hang_full_structured_3d)
UNSUPPORTED(solver_refine_operator_3d)
UNSUPPORTED(solver_coarsen_operator_3d)
UNSUPPORTED(solver_residual_bc_unstructured)
UNSUPPORTED(solver_residual_face_full_unstructured)
UNSUPPORTED(solver_residual_face_hang_unstructured_2d)
UNSUPPORTED(solver_residual_face_hang_unstructured_3d)
