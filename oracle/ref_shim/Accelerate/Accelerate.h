/* Stand-in for Apple's <Accelerate/Accelerate.h> so that the reference's
 * headers compile on Linux.  The reference only uses the three LAPACK
 * routines it declares itself (helpers.h:15-19); they are provided by
 * lapack_shim.c in this directory.  Test infrastructure only. */
#pragma once
