// Host-only part of the C ABI: loading a system through the drop-in readers and
// inspecting its topology (no GPU needed).
#include <cmath>
#include <cstring>
#include <new>

#include "host.h"

using namespace fz;

extern "C" fz_status fz_load_system(const fz_config* cfg, fz_system** out) {
  if (!cfg || !out) return fail(FZ_ERR_ARG, "fz_load_system: null argument");
  *out = nullptr;
  fz_system* s = new (std::nothrow) fz_system();
  if (!s) return fail(FZ_ERR_NOMEM, "host allocation failed");
  s->cfg = *cfg;
  fz_status st;
  // LoadCoord -> ReadPsf_CHARMM -> ReadPrm_CHARMM -> build_constraints -> GenExcl_minimal_new
  if ((st = read_coordinates(cfg->coordinates, s->top)) != FZ_OK ||
      (st = read_psf(cfg->structure, cfg->topology, *cfg, s->top)) != FZ_OK ||
      (st = read_prm(cfg->parameters, s->top)) != FZ_OK || (st = build_constraints(*cfg, s->top)) != FZ_OK ||
      (st = build_exclusions(s->top, cfg->kappa)) != FZ_OK) {
    delete s;
    return st;
  }
  *out = s;
  return FZ_OK;
}

extern "C" fz_status fz_get_info(const fz_system* s, fz_info* o) {
  if (!s || !o) return fail(FZ_ERR_ARG, "fz_get_info: null argument");
  const Topology& t = s->top;
  std::memset(o, 0, sizeof(*o));
  o->natom = t.n;
  o->ntypes = (int)t.type_names.size();
  o->nbond = (int)t.bond_k.size();
  o->nangle = (int)t.angle_k.size();
  o->nureyb = (int)t.ub_k.size();
  o->ndihedral = (int)t.psf_dihe.size() / 4;
  o->nimproper = (int)t.impr_k.size();
  o->nconstraint = (int)t.cons_d.size();
  o->ncluster = (int)t.clusters.size();
  o->nexcl_pairs = (int)t.excl_pairs.size() / 2;
  o->n14_pairs = (int)t.p14_pairs.size() / 2;
  o->ndihedral_terms = (int)t.dihe_k.size();
  for (int k = 0; k < 3; ++k) {
    o->pme_grid[k] = s->cfg.pme_grid[k];
    o->box[k] = s->cfg.box[k];
  }
  return FZ_OK;
}

template <class T>
static fz_status copy_vec(const std::vector<T>& v, void* out, size_t bytes, const char* name) {
  if (bytes != v.size() * sizeof(T))
    return fail(FZ_ERR_ARG, std::string("fz_get_array(") + name + "): expected " + std::to_string(v.size() * sizeof(T)) +
                                " bytes");
  if (!v.empty()) std::memcpy(out, v.data(), bytes);
  return FZ_OK;
}

extern "C" fz_status fz_get_array(const fz_system* s, const char* name, void* out, size_t bytes) {
  if (!s || !name || (!out && bytes)) return fail(FZ_ERR_ARG, "fz_get_array: null argument");
  const Topology& t = s->top;
  const std::string n(name);
#define FZ_ARR(key, vec) \
  if (n == key) return copy_vec(t.vec, out, bytes, name);
  FZ_ARR("pos", pos) FZ_ARR("q", q) FZ_ARR("mass", mass) FZ_ARR("type", type) FZ_ARR("eps4", eps4)
  FZ_ARR("sig2", sig2) FZ_ARR("eps4_14", eps4_14) FZ_ARR("sig2_14", sig2_14) FZ_ARR("bond", bond)
  FZ_ARR("bond_k", bond_k) FZ_ARR("bond_r0", bond_r0) FZ_ARR("angle", angle) FZ_ARR("angle_k", angle_k)
  FZ_ARR("angle_t0", angle_t0) FZ_ARR("ureyb", ub) FZ_ARR("ureyb_k", ub_k) FZ_ARR("ureyb_r0", ub_r0)
  FZ_ARR("dihe", dihe) FZ_ARR("dihe_k", dihe_k) FZ_ARR("dihe_n", dihe_n) FZ_ARR("dihe_d", dihe_d)
  FZ_ARR("impr", impr) FZ_ARR("impr_k", impr_k) FZ_ARR("impr_p0", impr_p0) FZ_ARR("cons", cons)
  FZ_ARR("cons_d", cons_d) FZ_ARR("excl", excl_pairs) FZ_ARR("p14", p14_pairs)
#undef FZ_ARR
  return fail(FZ_ERR_ARG, "fz_get_array: unknown array " + n);
}

extern "C" fz_status fz_free(fz_system* s) {
  if (!s) return FZ_OK;
  if (s->eng) destroy_engine(s->eng);
  delete s;
  return FZ_OK;
}
