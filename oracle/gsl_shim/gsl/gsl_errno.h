/* Minimal GSL-compatible error codes for building the reference's hot-path
 * sources without GNU GSL (which is absent from this image).  Test
 * infrastructure only: written from the GSL API documentation, no GSL source. */
#ifndef WRT_GSL_SHIM_ERRNO_H
#define WRT_GSL_SHIM_ERRNO_H
#define GSL_SUCCESS 0
#define GSL_FAILURE (-1)
#define GSL_EDOM 1
#define GSL_EINVAL 4
#define GSL_ENOMEM 8
#endif
