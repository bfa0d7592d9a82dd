/* Empty (test infrastructure, oracle/build_ref.py): see accfft.h. */
#pragma once
