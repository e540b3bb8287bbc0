/* Empty stand-in for the TI C7000 compiler's <c7x.h>.
 * The reference's natural-C (_cn) sources include <c7x.h> only through
 * src/common/FFTLIB_types.h; none of the declarations they use come from it.
 * This file lets those sources compile with the host gcc. Test infrastructure. */
#ifndef ORACLE_SHIM_C7X_SCALABLE_H
#define ORACLE_SHIM_C7X_SCALABLE_H
#endif
