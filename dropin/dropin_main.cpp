/*
 * dropin_main.cpp -- the reference's unchanged main program (vie_fft/CG_FFT_VIE.cpp
 * with Model.h, NearFar.h and ReadFile.h) built on the drop-in headers.
 *
 * The drop-in GreenFunction.h, fft.h and CG_Iteration.h are included first;
 * they define the reference's include guards, so when CG_FFT_VIE.cpp includes
 * the reference's own copies those are skipped.  A maintainer can instead copy
 * the three headers (and mkl.h) over the reference's in vie_fft/.
 */
#include "GreenFunction.h"
#include "fft.h"
#include "CG_Iteration.h"
#include "CG_FFT_VIE.cpp"
