// C ABI of the propagation pieces: orbital exponential propagator and the
// Loewdin re-orthonormalisation.
#include "context.hpp"
#include "../../include/sincgpu.h"

using namespace sincgpu;

extern "C" {

int sincgpu_orbprop_setup(sincgpu_ctx* h, int expodim, int maxexpodim, double expostepfac,
                          double first_stepsize) {
  CTX_CHECK(h);
  SG_CHECK(expodim >= 1 && maxexpodim >= 1 && maxexpodim <= 125, SINCGPU_EINVAL,
           "expodim %d / maxexpodim %d outside [1,125]", expodim, maxexpodim);
  SG_CHECK(first_stepsize > 0 && expostepfac > 0, SINCGPU_EINVAL, "step parameters must be positive");
  OrbPropState s;
  s.expodim = expodim;
  s.maxexpodim = maxexpodim;
  s.expostepfac = expostepfac;
  s.first_stepsize = first_stepsize;
  h->c.orb = s;
  return SINCGPU_OK;
}

int sincgpu_orbprop_state(sincgpu_ctx* h, int* thisexpodim, double* tempstepsize, int* exposet, int* icalled) {
  CTX_CHECK(h);
  const OrbPropState& s = h->c.orb;
  if (thisexpodim) *thisexpodim = s.thisexpodim;
  if (tempstepsize) *tempstepsize = s.tempstepsize;
  if (exposet) *exposet = s.exposet;
  if (icalled) *icalled = s.icalled;
  return SINCGPU_OK;
}

int sincgpu_expospfprop_dev(sincgpu_ctx* h, double* phi, const double* denmat0, const double* invdenmat0,
                            const double* reducedpot0, const double* denmat1, const double* invdenmat1,
                            const double* reducedpot1, double tin, double tout, double firsttime,
                            double lasttime, int linearflag, double tre, double tim, double ezfield,
                            double expotol, int* numiters) {
  CTX_CHECK(h);
  SG_CHECK(phi && denmat0 && invdenmat0 && reducedpot0, SINCGPU_EINVAL, "null argument");
  SG_CHECK(!linearflag || (denmat1 && invdenmat1 && reducedpot1), SINCGPU_EINVAL,
           "the linear blend needs both mean-field slots");
  MeanFieldSlot slots[2] = {
      {(const double2*)denmat0, (const double2*)invdenmat0, (const double2*)reducedpot0},
      {(const double2*)denmat1, (const double2*)invdenmat1, (const double2*)reducedpot1}};
  return expospfprop(h->c, (double2*)phi, slots, tin, tout, firsttime, lasttime, linearflag != 0,
                     make_double2(tre, tim), ezfield, expotol, numiters);
}

int sincgpu_spf_orthogit_dev(sincgpu_ctx* h, double* phi, double* error) {
  CTX_CHECK(h);
  SG_CHECK(phi, SINCGPU_EINVAL, "null argument");
  return spf_orthogit(h->c, (double2*)phi, error);
}

}  // extern "C"
