/* Stand-in for the absent CFITSIO header (oracle build only).  FITS I/O is
   not on the ray-shooting path; every routine is a no-op returning 0. */
#pragma once
typedef struct fitsfile_ fitsfile;
#define FLEN_CARD 81
#define FLEN_VALUE 71
#define FLEN_KEYWORD 75
#define FLEN_COMMENT 73
#define FLEN_ERRMSG 81
#define TFLOAT 1
#define TDOUBLE 2
#define READONLY 3
#define FLOAT_IMG 4
#define DOUBLE_IMG 5
#define TLONG 6
#define TULONG 7
#define TINT 8
#define TSTRING 9
#define SHORT_IMG 10
#define READWRITE 11
#define LONG_IMG 12
#define LONGLONG_IMG 13
#define BYTE_IMG 14
#define BINARY_TBL 15
#define ASCII_TBL 16
#define IMAGE_HDU 17
#define TSHORT 18
#define TUINT 19
#define TLONGLONG 20
#define TBYTE 21
#define TLOGICAL 22
#define TUSHORT 23
#define TSBYTE 24
#define KEY_NO_EXIST 25
#define END_OF_FILE 26
#define ANY_HDU 27
#define CASEINSEN 28
#define CASESEN 29
inline int fits_write_pix(...) { return 0; }
inline int fits_create_img(...) { return 0; }
inline int fits_read_pix(...) { return 0; }
inline int fits_read_col(...) { return 0; }
inline int fits_open_image(...) { return 0; }
inline int fits_update_key(...) { return 0; }
inline int fits_read_key(...) { return 0; }
inline int fits_close_file(...) { return 0; }
inline int fits_read_col_flt(...) { return 0; }
inline int fits_read_subset(...) { return 0; }
inline int fits_movabs_hdu(...) { return 0; }
inline int fits_get_num_hdus(...) { return 0; }
inline int fits_get_hdu_num(...) { return 0; }
inline int fits_get_hdrspace(...) { return 0; }
inline int fits_create_file(...) { return 0; }
inline int fits_write_record(...) { return 0; }
inline int fits_write_key(...) { return 0; }
inline int fits_report_error(...) { return 0; }
inline int fits_read_record(...) { return 0; }
inline int fits_parse_value(...) { return 0; }
inline int fits_open_table(...) { return 0; }
inline int fits_open_file(...) { return 0; }
inline int fits_movrel_hdu(...) { return 0; }
inline int fits_get_num_rows(...) { return 0; }
inline int fits_get_num_cols(...) { return 0; }
inline int fits_get_keytype(...) { return 0; }
inline int fits_get_img_type(...) { return 0; }
inline int fits_get_img_size(...) { return 0; }
inline int fits_get_img_dim(...) { return 0; }
inline int fits_get_hdu_type(...) { return 0; }
inline int fits_get_coltype(...) { return 0; }
inline int fits_get_colnum(...) { return 0; }
inline int fits_get_colname(...) { return 0; }
inline int fits_delete_file(...) { return 0; }
inline int fits_write_col(...) { return 0; }
inline int fits_create_tbl(...) { return 0; }
inline int fits_insert_rows(...) { return 0; }
inline int fits_get_errstatus(...) { return 0; }
inline int fits_read_img(...) { return 0; }
inline int fits_write_img(...) { return 0; }
