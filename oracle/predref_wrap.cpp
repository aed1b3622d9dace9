// predref_wrap.cpp -- exposes the reference's own predicates.h, compiled for
// the host, to the tests (TEST INFRASTRUCTURE ONLY; the product never links
// it).  Built by oracle/ref_build.sh into oracle/_ref/libpredref.so from the
// header where it lies in the reference tree; nothing of it is copied here.
#define __device__
#include "predicates.h"

extern "C" {
void ref_exactinit(void) { exactinit(); }
float ref_orient3d(float *pa, float *pb, float *pc, float *pd) { return orient3d(pa, pb, pc, pd); }
float ref_insphere_w(float *pa, float *pb, float *pc, float *pd, float *pe, float wa, float wb,
                     float wc, float wd, float we) {
    return insphere_w(pa, pb, pc, pd, pe, wa, wb, wc, wd, we);
}
float ref_orient3d_l_w(float *p0, float *p1, float *p2, float *p3, float w0, float w1, float w2,
                       float w3, int lifted) {
    return orient3D_l_w(p0, p1, p2, p3, w0, w1, w2, w3, lifted != 0);
}
// The reference's SoS never returns when all 48 minors vanish; callers must
// not pass fully degenerate point sets (equal points with equal weights).
float ref_sos4(float *p0, float *p1, float *p2, float *p3, float *p4, float w0, float w1,
               float w2, float w3, float w4, int i0, int i1, int i2, int i3, int i4) {
    return orientation4SoS_w(p0, p1, p2, p3, p4, w0, w1, w2, w3, w4, i0, i1, i2, i3, i4);
}
}
