/* Empty (test infrastructure, oracle/build_ref.py): src/interp3.cpp includes
 * petsc.h only for PETSC_USE_REAL_SINGLE, which the recipe sets on the
 * command line for the single-precision build. */
#pragma once
