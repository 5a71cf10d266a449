// Restart files: SaveCheckpointBinary / LoadCheckpointBinary and SaveCheckpointAscii /
// LoadCheckpointAscii (src/prmwrite.cu:31-252), the same two layouts so restart files
// move between the reference and this library:
//   binary: int natom, int step, double seed, float box[3], float box_velocity[3],
//           then natom x (float x, y, z, vx, vy, vz)
//   ascii:  "%12d \n" natom, "%12d \n" step, "%le \n" seed,
//           "%12f %12f %12f %12f %12f %12f\n" box and box velocity,
//           natom lines "%10f %10f %10f %10f %10f %10f\n" (positions, velocities)
// Velocities are in A per AKMA time unit; the box velocity is the barostat's edge
// velocity (zero at constant volume).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "engine.h"

using namespace fz;

static int pick_format(const fz_system* s, int format) {
  if (format == 'a' || format == 'b') return format;
  return s->cfg.checkpointformat == 'a' ? 'a' : 'b';
}

extern "C" fz_status fz_checkpoint_save(fz_system* s, const char* path, int format) {
  if (!s || !path) return fail(FZ_ERR_ARG, "null argument");
  if (!s->eng) return fail(FZ_ERR_STATE, "fz_upload has not been called");
  Engine* e = s->eng;
  const int n = e->n;
  std::vector<float> pos(3 * (size_t)n), vel(3 * (size_t)n);
  fz_status r;
  if ((r = fz_get_state_f32(s, pos.data(), vel.data()))) return r;
  const int fmt = pick_format(s, format);
  const int step = (int)e->step;
  const double seed = (double)e->seed;
  float box[3], bvel[3];
  for (int d = 0; d < 3; ++d) {
    box[d] = (float)e->box_d[d];
    bvel[d] = e->npt ? (float)(e->Ldot * e->ratio[d]) : 0.f;
  }
  FILE* f = std::fopen(path, fmt == 'a' ? "w" : "wb");
  if (!f) return fail(FZ_ERR_IO, std::string("cannot write ") + path);
  bool ok = true;
  if (fmt == 'b') {
    ok = std::fwrite(&n, sizeof n, 1, f) == 1 && std::fwrite(&step, sizeof step, 1, f) == 1 &&
         std::fwrite(&seed, sizeof seed, 1, f) == 1 && std::fwrite(box, sizeof box, 1, f) == 1 &&
         std::fwrite(bvel, sizeof bvel, 1, f) == 1;
    for (int i = 0; ok && i < n; ++i) {
      const float rec[6] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]};
      ok = std::fwrite(rec, sizeof rec, 1, f) == 1;
    }
  } else {
    std::fprintf(f, "%12d \n%12d \n%le \n", n, step, seed);
    std::fprintf(f, "%12f %12f %12f %12f %12f %12f\n", box[0], box[1], box[2], bvel[0], bvel[1], bvel[2]);
    for (int i = 0; i < n; ++i)
      std::fprintf(f, "%10f %10f %10f %10f %10f %10f\n", pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], vel[3 * i],
                   vel[3 * i + 1], vel[3 * i + 2]);
    ok = !std::ferror(f);
  }
  if (std::fclose(f) != 0) ok = false;
  return ok ? FZ_OK : fail(FZ_ERR_IO, std::string("write error on ") + path);
}

extern "C" fz_status fz_checkpoint_load(fz_system* s, const char* path, int format) {
  if (!s || !path) return fail(FZ_ERR_ARG, "null argument");
  if (!s->eng) return fail(FZ_ERR_STATE, "fz_upload has not been called");
  Engine* e = s->eng;
  const int fmt = pick_format(s, format);
  FILE* f = std::fopen(path, fmt == 'a' ? "r" : "rb");
  if (!f) return fail(FZ_ERR_IO, std::string("cannot open ") + path);
  int n = 0, step = 0;
  double seed = 0;
  float box[3], bvel[3];
  std::vector<float> pos, vel;
  bool ok;
  if (fmt == 'b') {
    ok = std::fread(&n, sizeof n, 1, f) == 1 && std::fread(&step, sizeof step, 1, f) == 1 &&
         std::fread(&seed, sizeof seed, 1, f) == 1 && std::fread(box, sizeof box, 1, f) == 1 &&
         std::fread(bvel, sizeof bvel, 1, f) == 1 && n == e->n;
    pos.resize(3 * (size_t)e->n);
    vel.resize(3 * (size_t)e->n);
    for (int i = 0; ok && i < n; ++i) {
      float rec[6];
      ok = std::fread(rec, sizeof rec, 1, f) == 1;
      for (int c = 0; ok && c < 3; ++c) {
        pos[3 * i + c] = rec[c];
        vel[3 * i + c] = rec[3 + c];
      }
    }
  } else {
    ok = std::fscanf(f, "%d %d %lf %f %f %f %f %f %f", &n, &step, &seed, &box[0], &box[1], &box[2], &bvel[0],
                     &bvel[1], &bvel[2]) == 9 && n == e->n;
    pos.resize(3 * (size_t)e->n);
    vel.resize(3 * (size_t)e->n);
    for (int i = 0; ok && i < n; ++i)
      ok = std::fscanf(f, "%f %f %f %f %f %f", &pos[3 * i], &pos[3 * i + 1], &pos[3 * i + 2], &vel[3 * i],
                       &vel[3 * i + 1], &vel[3 * i + 2]) == 6;
  }
  std::fclose(f);
  if (!ok) {
    if (n != e->n && n > 0)
      return fail(FZ_ERR_PARSE, std::string(path) + ": restart file holds " + std::to_string(n) +
                                    " atoms, the system " + std::to_string(e->n));
    return fail(FZ_ERR_PARSE, std::string(path) + ": truncated or malformed restart file");
  }
  for (int d = 0; d < 3; ++d)
    if (!(box[d] > 0.f)) return fail(FZ_ERR_PARSE, std::string(path) + ": non-positive box edge");
  fz_status r;
  cudaSetDevice(e->dev);
  // a different box (a restart of a constant-pressure run) moves the engine to it
  if (std::fabs(box[0] - e->box_d[0]) > 1e-6 * e->box_d[0]) {
    for (int d = 1; d < 3; ++d)
      if (std::fabs(box[d] / box[0] - e->ratio[d]) > 1e-5)
        return fail(FZ_ERR_PARSE, std::string(path) + ": box aspect ratios differ from the system's");
    e->drop_graph();
    if ((r = set_box(e, box[0]))) return r;
  }
  if (e->npt) e->Ldot = bvel[0];
  e->step = step;
  e->seed = (unsigned long long)(long long)seed;
  return fz_set_state_f32(s, pos.data(), vel.data());
}
