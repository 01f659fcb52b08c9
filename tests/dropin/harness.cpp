// Test harness for the drop-in classes (pawan_b200/dropin): builds the
// reference's own wakes and integrators (compiled from the reference sources)
// around pawan::__cuda and pawan::__cuda_rk4, and runs them side by side with
// the reference's __interaction.  Built by `make -C oracle dropin` into
// oracle/_ref/libpawan_dropin.so; used only by tests/test_gpu_dropin.py.
#include <cstdio>
#include <string>
#include <vector>

#include "pawan_b200/dropin/cuda_interaction.h"
#include "src/integration/rk4.h"
#include "src/interaction/interaction.h"
#include "src/io/io.h"
#include "src/resolve/resolve.h"
#include "src/wake/vring.h"

namespace {

class ArrayWake : public pawan::__wake {
 public:
  ArrayWake(size_t n, const double *pos, const double *vor, const double *rad, const double *vol) {
    gsl_matrix_free(_position);
    gsl_matrix_free(_velocity);
    gsl_matrix_free(_vorticity);
    gsl_matrix_free(_retvorcity);
    gsl_vector_free(_radius);
    gsl_vector_free(_volume);
    gsl_vector_free(_birthstrength);
    gsl_matrix_free(_vorticityfield);
    create_particles((int)n);
    for (size_t i = 0; i < n; ++i) {
      for (size_t d = 0; d < 3; ++d) {
        gsl_matrix_set(_position, i, d, pos[3 * i + d]);
        gsl_matrix_set(_vorticity, i, d, vor[3 * i + d]);
      }
      gsl_vector_set(_radius, i, rad[i]);
      gsl_vector_set(_volume, i, vol[i]);
    }
  }
};

class NuInteraction : public pawan::__interaction {
 public:
  explicit NuInteraction(double nu) { _nu = nu; }
  void read(double *out) const {
    for (int d = 0; d < 3; ++d) {
      out[d] = gsl_vector_get(_totalVorticity, d);
      out[3 + d] = gsl_vector_get(_linearImpulse, d);
      out[6 + d] = gsl_vector_get(_angularImpulse, d);
    }
    out[9] = _enstrophy;
    out[10] = _helicity;
  }
};

class ReadCuda : public pawan::__cuda {
 public:
  using pawan::__cuda::__cuda;
  void read(double *out) const {
    for (int d = 0; d < 3; ++d) {
      out[d] = gsl_vector_get(_totalVorticity, d);
      out[3 + d] = gsl_vector_get(_linearImpulse, d);
      out[6 + d] = gsl_vector_get(_angularImpulse, d);
    }
    out[9] = _enstrophy;
    out[10] = _helicity;
  }
};

class StepRK4 : public pawan::__rk4 {
 public:
  StepRK4() : pawan::__rk4(1.0, 1) {}
  void run(double dt, pawan::__system *S, gsl_vector *st) { step(dt, S, st); }
};

class StepCudaRK4 : public pawan::__cuda_rk4 {
 public:
  StepCudaRK4() : pawan::__cuda_rk4(1.0, 1) {}
  void run(double dt, pawan::__system *S, gsl_vector *st) { step(dt, S, st); }
};

std::vector<pawan::__wake *> make_wakes(int nw, const size_t *counts, const double *pos,
                                        const double *vor, const double *rad, const double *vol) {
  std::vector<pawan::__wake *> W;
  size_t o = 0;
  for (int w = 0; w < nw; ++w) {
    W.push_back(new ArrayWake(counts[w], pos + 3 * o, vor + 3 * o, rad + o, vol + o));
    o += counts[w];
  }
  return W;
}

ReadCuda *make_cuda(std::vector<pawan::__wake *> &W, double nu, int precision) {
  ReadCuda *C = new ReadCuda(W[0], nu, precision, 0);
  for (size_t k = 1; k < W.size(); ++k) C->addWake(W[k]);
  return C;
}

}  // namespace

extern "C" {

// rates (6N, reference layout) of one solve(): by __cuda (gpu) and by the
// reference __interaction (cpu).  Returns 0 on success.
int dropin_solve(int nw, const size_t *counts, const double *pos, const double *vor,
                 const double *rad, const double *vol, double nu, int precision, double *gpu,
                 double *cpu) {
  try {
    auto Wg = make_wakes(nw, counts, pos, vor, rad, vol);
    auto Wc = make_wakes(nw, counts, pos, vor, rad, vol);
    ReadCuda *G = make_cuda(Wg, nu, precision);
    NuInteraction *R = new NuInteraction(nu);
    for (auto *w : Wc) R->addWake(w);
    G->solve();
    R->solve();
    gsl_vector_view vg = gsl_vector_view_array(gpu, G->_size);
    gsl_vector_view vc = gsl_vector_view_array(cpu, R->_size);
    G->getRates(&vg.vector);
    R->getRates(&vc.vector);
    delete G;
    delete R;
    for (auto *w : Wg) delete w;
    for (auto *w : Wc) delete w;
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}

// nsteps RK4 of `state` (6N, in/out) with: mode 0 = reference __rk4 driving
// __cuda (host path, 4 GPU solves per step); mode 1 = __cuda_rk4 driving
// __cuda (device-resident); mode 2 = reference __rk4 driving __interaction.
int dropin_rk4(int nw, const size_t *counts, const double *pos, const double *vor,
               const double *rad, const double *vol, double nu, int precision, double dt,
               size_t nsteps, int mode, double *state) {
  try {
    auto W = make_wakes(nw, counts, pos, vor, rad, vol);
    pawan::__interaction *S;
    if (mode == 2) {
      NuInteraction *R = new NuInteraction(nu);
      for (auto *w : W) R->addWake(w);
      S = R;
    } else {
      S = make_cuda(W, nu, precision);
    }
    gsl_vector_view v = gsl_vector_view_array(state, S->_size);
    if (mode == 1) {
      StepCudaRK4 rk;
      for (size_t i = 0; i < nsteps; ++i) rk.run(dt, S, &v.vector);
    } else {
      StepRK4 rk;
      for (size_t i = 0; i < nsteps; ++i) rk.run(dt, S, &v.vector);
    }
    if (mode == 2) delete static_cast<NuInteraction *>(S);
    else delete static_cast<ReadCuda *>(S);
    for (auto *w : W) delete w;
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}

// diagnose() of __cuda (gpu[11]) and of the reference (cpu[11]).
int dropin_diagnose(int nw, const size_t *counts, const double *pos, const double *vor,
                    const double *rad, const double *vol, double *gpu, double *cpu) {
  try {
    auto Wg = make_wakes(nw, counts, pos, vor, rad, vol);
    auto Wc = make_wakes(nw, counts, pos, vor, rad, vol);
    ReadCuda *G = make_cuda(Wg, 0.0, PAWAN_PREC_F32);
    NuInteraction *R = new NuInteraction(0.0);
    for (auto *w : Wc) R->addWake(w);
    G->diagnose();
    R->diagnose();
    G->read(gpu);
    R->read(cpu);
    delete G;
    delete R;
    for (auto *w : Wg) delete w;
    for (auto *w : Wc) delete w;
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}

// __cuda_rk4(T, n).integrate(__cuda) through the reference's non-virtual
// integrate() (an __integration pointer: host loop, frames from the wakes; mode
// 0) or through __cuda_rk4::integrate (device loop, asynchronous frames; mode
// 1) -- writes data/temp.wake under the cwd.
int dropin_integrate2(int nw, const size_t *counts, const double *pos, const double *vor,
                      const double *rad, const double *vol, double nu, int precision, double T,
                      size_t n, int mode) {
  try {
    auto W = make_wakes(nw, counts, pos, vor, rad, vol);
    ReadCuda *G = make_cuda(W, nu, precision);
    pawan::__io io;
    pawan::__cuda_rk4 rk(T, n);
    if (mode == 1)
      rk.integrate(G, &io);
    else
      static_cast<pawan::__integration &>(rk).integrate(G, &io);
    delete G;
    for (auto *w : W) delete w;
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}

// __cuda_rk4(T, n).integrate(__cuda) -- writes data/temp.wake under the cwd.
int dropin_integrate(int nw, const size_t *counts, const double *pos, const double *vor,
                     const double *rad, const double *vol, double nu, int precision, double T,
                     size_t n) {
  try {
    auto W = make_wakes(nw, counts, pos, vor, rad, vol);
    ReadCuda *G = make_cuda(W, nu, precision);
    pawan::__io io;
    pawan::__cuda_rk4 rk(T, n);
    rk.integrate(G, &io);
    delete G;
    for (auto *w : W) delete w;
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}

// Vorticity field (N x 3, wake order) after resolve(): __cuda (gpu) and the
// reference __interaction (cpu).
int dropin_influence(int nw, const size_t *counts, const double *pos, const double *vor,
                     const double *rad, const double *vol, double *gpu, double *cpu) {
  try {
    auto Wg = make_wakes(nw, counts, pos, vor, rad, vol);
    auto Wc = make_wakes(nw, counts, pos, vor, rad, vol);
    ReadCuda *G = make_cuda(Wg, 0.0, PAWAN_PREC_F32);
    NuInteraction *R = new NuInteraction(0.0);
    for (auto *w : Wc) R->addWake(w);
    G->resolve();
    R->resolve();
    size_t o = 0;
    for (size_t k = 0; k < Wg.size(); ++k) {
      for (size_t i = 0; i < Wg[k]->_numParticles; ++i)
        for (size_t d = 0; d < 3; ++d) {
          gpu[3 * (o + i) + d] = gsl_matrix_get(Wg[k]->_vorticityfield, i, d);
          cpu[3 * (o + i) + d] = gsl_matrix_get(Wc[k]->_vorticityfield, i, d);
        }
      o += Wg[k]->_numParticles;
    }
    delete G;
    delete R;
    for (auto *w : Wg) delete w;
    for (auto *w : Wc) delete w;
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}

// The reference's __resolve::rebuild on a __vring(radius, core, layers):
// driven through __cuda (gpu) and through the reference __interaction (cpu).
// Writes data/temp.wakeinfluence under the cwd (twice).  The resolved
// strength vectors (length (2 layers + 1)^2) land in gpu / cpu.
int dropin_vring_resolve(double radius, double core, int layers, double *gpu, double *cpu) {
  try {
    pawan::__vring *Vg = new pawan::__vring(radius, core, layers);
    pawan::__vring *Vc = new pawan::__vring(radius, core, layers);
    ReadCuda *G = new ReadCuda(Vg, 0.0, PAWAN_PREC_F32, 0);
    NuInteraction *R = new NuInteraction(0.0);
    R->addWake(Vc);
    pawan::__io io;
    pawan::__resolve rs;
    rs.rebuild(G, &io);
    rs.rebuild(R, &io);
    gsl_vector_view vg = gsl_vector_view_array(gpu, G->_size);
    gsl_vector_view vc = gsl_vector_view_array(cpu, R->_size);
    G->getStates(&vg.vector);
    R->getStates(&vc.vector);
    delete G;
    delete R;
    delete Vg;
    delete Vc;
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}

static std::vector<char> file_bytes(const std::string &path) {
  std::vector<char> out;
  FILE *f = std::fopen(path.c_str(), "rb");
  if (!f) return out;
  char buf[1 << 16];
  size_t r;
  while ((r = std::fread(buf, 1, sizeof buf, f)) > 0) out.insert(out.end(), buf, buf + r);
  std::fclose(f);
  return out;
}

// __cuda_resolve::rebuild (influence-matrix columns batched on the device)
// against the reference's __resolve::rebuild, both over a __cuda on a
// __vring(radius, core, layers).  Resolved strengths into batched / percol;
// *same_file = 1 when the two .wakeinfluence files are byte-identical.
int dropin_vring_resolve_batched(double radius, double core, int layers, double *batched,
                                 double *percol, int *same_file) {
  try {
    pawan::__vring *Vb = new pawan::__vring(radius, core, layers);
    pawan::__vring *Vp = new pawan::__vring(radius, core, layers);
    ReadCuda *B = new ReadCuda(Vb, 0.0, PAWAN_PREC_F32, 0);
    ReadCuda *P = new ReadCuda(Vp, 0.0, PAWAN_PREC_F32, 0);
    pawan::__io io;
    const std::string path = io.getFile() + ".wakeinfluence";
    pawan::__cuda_resolve batched_resolve;
    batched_resolve.rebuild(B, &io);
    const std::vector<char> fb = file_bytes(path);
    pawan::__resolve reference_resolve;
    reference_resolve.rebuild(P, &io);
    const std::vector<char> fp = file_bytes(path);
    *same_file = (!fb.empty() && fb == fp) ? 1 : 0;
    gsl_vector_view vb = gsl_vector_view_array(batched, B->_size);
    gsl_vector_view vp = gsl_vector_view_array(percol, P->_size);
    B->getStates(&vb.vector);
    P->getStates(&vp.vector);
    delete B;
    delete P;
    delete Vb;
    delete Vp;
    return 0;
  } catch (const std::exception &e) {
    std::fprintf(stderr, "%s\n", e.what());
    return 1;
  }
}

}  // extern "C"
