/*
 * fitsio.h -- minimal stand-in for the cfitsio header, written for this project.
 *
 * TEST INFRASTRUCTURE ONLY. It exists so that the reference's own
 * gpair1/trunk/cpu.c and gpair1/trunk/getoifits.c compile unchanged into the
 * oracle library (oracle/_ref). cfitsio itself is not installed; the few
 * fits_* entry points those two files call are implemented in memory by
 * oifits_mem.c (no file I/O).
 *
 * Only names, constant values and signatures of the public cfitsio API
 * are declared here.
 */
#ifndef GPAIR_ORACLE_FITSIO_SHIM_H
#define GPAIR_ORACLE_FITSIO_SHIM_H

#include <stdio.h>

#define FLEN_FILENAME 1025
#define FLEN_KEYWORD 75
#define FLEN_CARD 81
#define FLEN_VALUE 71
#define FLEN_COMMENT 73
#define FLEN_ERRMSG 81

#define READONLY 0
#define READWRITE 1

#define IMAGE_HDU 0
#define ASCII_TBL 1
#define BINARY_TBL 2

#define TLOGICAL 14
#define TSTRING 16
#define TSHORT 21
#define TINT 31
#define TLONG 41
#define TFLOAT 42
#define TDOUBLE 82

#define DOUBLE_IMG (-64)
#define FLOAT_IMG (-32)

#define CASEINSEN 0
#define KEY_NO_EXIST 202
#define END_OF_FILE 107
#define BAD_HDU_NUM 301

typedef struct oracle_fitsfile fitsfile;

int fits_open_file(fitsfile **fptr, const char *name, int mode, int *status);
int fits_close_file(fitsfile *fptr, int *status);
void fits_report_error(FILE *stream, int status);
int fits_movabs_hdu(fitsfile *fptr, int hdunum, int *hdutype, int *status);
int fits_movrel_hdu(fitsfile *fptr, int nmove, int *hdutype, int *status);
int fits_get_hdu_num(fitsfile *fptr, int *hdunum);
int fits_get_num_hdus(fitsfile *fptr, int *nhdu, int *status);
int fits_read_key(fitsfile *fptr, int datatype, const char *keyname, void *value, char *comment, int *status);

#endif
