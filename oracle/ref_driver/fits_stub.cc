// Stand-ins for the three FITS entry points of the reference's cmlib/fits_read.h.
// The reference links cfitsio for them (cmlib/fits_read.cc); cfitsio is not
// installed here and no part of the synthesis / response / fit path reads FITS,
// so the oracle build replaces them with functions that report "unsupported".
// Test infrastructure only: compiled into oracle/_ref by oracle/Makefile.
#include <stdio.h>
#include "types.h"
#include "io.h"
#include "fits_read.h"

byte *fits_read(char *file_name, int *&ds, int &nd, char *&header, int &type, io_class &io)
{
  fprintf(stderr, "oracle build: FITS input (%s) is not supported\n", file_name);
  ds = 0; nd = 0; header = 0; type = 0;
  return 0;
}

int fits_data_type(const char *file_name, io_class &io)
{
  fprintf(stderr, "oracle build: FITS input (%s) is not supported\n", file_name);
  return -1;
}

int fits_write_4d_fpt(char *filename, fp_t ****)
{
  fprintf(stderr, "oracle build: FITS output (%s) is not supported\n", filename);
  return -1;
}
