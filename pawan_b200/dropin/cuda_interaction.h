/* Drop-in GPU interaction for pawan.
 *
 * pawan::__cuda is a sibling of the reference's OpenMP class pawan::__parallel
 * (src/interaction/parallel.h:20-145): same constructors (one or two wakes,
 * more through addWake), same __system / __interaction interface, so the
 * reference's integrators (__integration, __rk4) drive it unchanged.  The
 * all-pairs interaction of every solve() runs on a B200 through the C ABI in
 * include/pawan_b200.h; results land in each wake's _velocity and _retvorcity
 * exactly where the reference's interact() puts them, so getRates() and the
 * rest of the reference code see no difference.
 *
 * pawan::__cuda_rk4 is a drop-in for __rk4 (src/integration/rk4.h:14-42): given
 * a __cuda system it runs whole RK4 steps on the device (state uploaded once
 * per step, the four stages and their updates in HBM, state read back once);
 * given any other __system it is the reference __rk4.
 *
 * Compile these two files inside the reference tree (they include its
 * headers) and link libpawan_b200.so.
 */
#ifndef PAWAN_B200_DROPIN_CUDA_INTERACTION_H
#define PAWAN_B200_DROPIN_CUDA_INTERACTION_H

#include <stdexcept>
#include <string>
#include <vector>

#include "pawan_b200.h"
#include "src/integration/rk4.h"
#include "src/interaction/interaction.h"
#include "src/resolve/resolve.h"
#include "src/wake/wake.h"

namespace pawan {

class __cuda : public __interaction {
 public:
  /* nu defaults to the reference's hard-coded 2.5e-3 (interaction.cpp:13). */
  explicit __cuda(__wake *W, double nu = 2.5e-3, int precision = PAWAN_PREC_F32, int device = 0);
  __cuda(__wake *W1, __wake *W2, double nu = 2.5e-3, int precision = PAWAN_PREC_F32,
         int device = 0);
  ~__cuda();

  void addWake(__wake *W) override;
  /* diagnose() of the reference (interaction.cpp:49-93), FP64 on the GPU; fills
   * the same members and prints the same lines. */
  void diagnose() override;

  double kineticEnergy();
  void setViscosity(double nu);
  /* The smoothing kernel the reference selects at compile time
   * (interaction_utils.h:13-24): PAWAN_KERNEL_HIGHORDER (its default) or
   * PAWAN_KERNEL_GAUSSIAN (src/interaction/gaussian.h). */
  void setKernel(int kernel);
  /* Uploads the wakes' current positions and vorticities (and, the first time
   * or after addWake, radii and volumes). */
  void upload();
  /* Copies the device state back into the wakes' _position / _vorticity. */
  void download();
  pawan_system *device_system() { return _sys; }
  /* Particles over all wakes; their current positions / vorticities as N x 3
   * rows in wake order; a field of that shape written into every wake's
   * _vorticityfield. */
  size_t numParticles() const;
  void gatherPositions(double *out) const;
  void gatherVorticity(double *out) const;
  void scatterField(const double *field);
  /* The vorticity field of ncols strength vectors (ncols x N x 3, wake order)
   * over the positions and radii last uploaded. */
  void influenceColumns(size_t ncols, const double *alpha, double *field);

 protected:
  /* The whole-solve hook (interaction.h:106): every wake pair in one launch. */
  void interact() override;
  /* The vorticity-field hook (interaction.h:112) behind resolve(): FP64 on the
   * device, into every wake's _vorticityfield, so the reference's
   * __resolve::rebuild (src/resolve/resolve.cpp:10-57) builds its influence
   * matrix on the GPU. */
  void influence() override;

 private:
  std::vector<__wake *> _wakes;
  pawan_ctx *_ctx = nullptr;
  pawan_system *_sys = nullptr;
  int _precision;
  int _device;
  int _kernel = PAWAN_KERNEL_HIGHORDER;
  bool _particles_uploaded = false;
  void ensure_system();
  void check(int status, const char *what) const;
};

/* pawan::__cuda_resolve is a drop-in for __resolve (src/resolve/resolve.h):
 * rebuild() does what the reference's does (resolve.cpp:10-57) -- the same
 * .wakeinfluence frames, the same influence matrix filled column by column
 * through the system's setStates / getRates, the same GSL LU solve, and
 * setStates of the result -- but the vorticity fields of the columns are
 * evaluated on the device in batches: consecutive columns whose states put
 * the particles at the same positions (every column of a __vring, whose state
 * is its strengths) go to the GPU in one call instead of one solve each.
 * rebuild() is not virtual in the reference, so call it through a
 * __cuda_resolve; an interaction that is not a __cuda goes through the
 * reference's rebuild. */
class __cuda_resolve : public __resolve {
 public:
  void rebuild(__interaction *IN, __io *IO);
};

class __cuda_rk4 : public __rk4 {
 public:
  __cuda_rk4(const double &t, const size_t &n) : __rk4(t, n) {}
  ~__cuda_rk4() = default;
  /* __integration::integrate (integration.cpp:16-35) for a __cuda system: the
   * n steps stay on the device and the .wake frames (same file, same bytes
   * layout) are written by a background thread while the next steps run; the
   * wakes hold the final state afterwards.  Any other system goes through the
   * reference's integrate().  integrate() is not virtual in the reference, so
   * call it through a __cuda_rk4 (not an __integration) pointer or reference. */
  void integrate(__system *S, __io *IO);

 protected:
  void step(const double &dt, __system *S, gsl_vector *state) override;
};

}  // namespace pawan

#endif
