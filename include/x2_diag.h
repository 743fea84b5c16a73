/* x2_diag.h — entry points of the diagnostic build of libx2 (libx2diag.so) only; the product library does not
 * export them. No counterpart in the reference: they serve the parity investigation of per-sample radiance against the
 * reference integrator.
 *
 * The transcendental functions of the per-sample kernels (x2_integrate) run either as CUDA's single-precision
 * functions (mode bit 0 clear, as in the product) or in double rounded to float (bit 0 set); with bit 1 set every
 * call (x2_diag_call: function, arguments, results) is appended to a device buffer of `capacity` records, in call
 * order when one sample is integrated a call. With bit 2 set the volume march's single scattering gives each distance
 * sample the light point of its pair's equi-angular sample (the pivot of both MIS weights) instead of a point of its
 * own: not the reference's estimator; a study of its bias. All act on the current device. */
#ifndef X2_DIAG_H
#define X2_DIAG_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct x2_diag_call {
    uint32_t fn;   /* 1 sincos, 2 exp, 3 log, 4 tan, 5 atan2, 6 pow, 7 acos, 8 cos */
    float a, b;    /* arguments (b: atan2's x, pow's exponent) */
    float r0, r1;  /* results (r1: sincos's cosine) */
} x2_diag_call;

int x2_diag_set(int mode, void* d_calls, uint32_t capacity);  /* also clears the record count */
int x2_diag_count(uint32_t* count);                           /* records appended so far (may exceed capacity) */

#ifdef __cplusplus
}
#endif
#endif
