/* Test-only stand-in for <mkl.h>: the marker step never reaches the PARDISO solve, so a no-op suffices. */
#define PARDISO(...) ((void)0)
