/* Empty stand-in for <mkl/mkl.h>: the reference includes it (src/general.cuh:6)
 * but calls no MKL symbol, and MKL is not installed. Used only when building
 * the reference sources into oracle/_ref/. */
