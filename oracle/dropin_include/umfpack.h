/* "umfpack.h" for the build of the reference drivers in
 * oracle/_ref/libgermaine_ref_dropin.so: the UMFPACK calls resolve to
 * libgermaine_umfpack.so.  Test infrastructure only. */
#include "germaine_umfpack.h"
