// C wrapper over the reference's HEALPix (src/Healpix_2.15a/healpix_base.cc),
// compiled from the reference sources into oracle/_ref/ to pin the HEALPix
// restatements of the oracle and of the product sampler.  Test infrastructure.
#include "src/Healpix_2.15a/healpix_base.h"

extern "C" void ref_hp_pix2zphi(int order, int ipix, double* z, double* phi)
{
    Healpix_Base b(order, NEST);
    b.pix2ang_z_phi(ipix, *z, *phi);
}

extern "C" int ref_hp_xyf2nest(int order, int x, int y, int face)
{
    Healpix_Base b(order, NEST);
    return b.xyf2nest(x, y, face);
}

extern "C" void ref_hp_nest2xyf(int order, int pix, int* x, int* y, int* face)
{
    Healpix_Base b(order, NEST);
    b.nest2xyf(pix, *x, *y, *face);
}

extern "C" double ref_hp_max_pixrad(int order)
{
    Healpix_Base b(order, NEST);
    return b.max_pixrad();
}
