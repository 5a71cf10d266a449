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

// ---------------------------------------------------------------- DCD trajectories
// The CHARMM DCD layout the reference writes through charmm_trj_write_header/titles/
// natoms/frame (src/io/charmmio.c, called from src/fenzi.cu:280-340, 513-528): Fortran
// unformatted records (int32 length, payload, int32 length).  Header record "CORD" +
// 20 int32 control words: frames, first step, output frequency, steps, 3 zeros,
// degrees-of-freedom word 1, fixed atoms 0, time step (float, AKMA units), unit cell
// flag 1, 4-D flag 0, charges flag 0, 6 zeros, version 34.  Then one 80-character
// title, the atom count, and per frame a unit-cell record of 6 doubles (A, 0, B, 0, 0,
// C for the rectangular box) and the X, Y, Z float records.
struct fz_dcd {
  fz_system* sys = nullptr;
  FILE* f = nullptr;
  int every = 1, frames = 0;
  std::vector<float> pos, buf;
};

static bool rec(FILE* f, const void* a, uint32_t na, const void* b = nullptr, uint32_t nb = 0) {
  const uint32_t len = na + nb;
  return std::fwrite(&len, 4, 1, f) == 1 && (na == 0 || std::fwrite(a, 1, na, f) == na) &&
         (nb == 0 || std::fwrite(b, 1, nb, f) == nb) && std::fwrite(&len, 4, 1, f) == 1;
}

static bool dcd_header(fz_dcd* d) {
  const fz_system* s = d->sys;
  uint32_t ctl[20] = {};
  ctl[0] = (uint32_t)d->frames;
  ctl[1] = (uint32_t)d->every;
  ctl[2] = (uint32_t)d->every;
  ctl[3] = (uint32_t)(d->frames * d->every);
  ctl[7] = 1;
  ctl[8] = 0;
  const float dt = (float)(s->cfg.timestep_ps / 4.888821e-2);  // ps -> AKMA time (src/fenzi.cu:320)
  std::memcpy(&ctl[9], &dt, 4);
  ctl[10] = 1;
  ctl[11] = 0;
  ctl[12] = 0;
  ctl[19] = 34;
  char title[80];
  std::memset(title, ' ', 80);
  const char* t = "Generated by fenzi_b200";
  std::memcpy(title, t, std::strlen(t));
  const int32_t ntitles = 1, natoms = s->top.n;
  return rec(d->f, "CORD", 4, ctl, sizeof ctl) && rec(d->f, &ntitles, 4, title, 80) && rec(d->f, &natoms, 4);
}

extern "C" fz_status fz_dcd_open(fz_system* s, const char* path, int every, fz_dcd** out) {
  if (!s || !path || !out) return fail(FZ_ERR_ARG, "null argument");
  if (!s->eng) return fail(FZ_ERR_STATE, "fz_upload has not been called");
  fz_dcd* d = new fz_dcd();
  d->sys = s;
  d->every = every > 0 ? every : 1;
  d->f = std::fopen(path, "wb");
  if (!d->f) {
    delete d;
    return fail(FZ_ERR_IO, std::string("cannot write ") + path);
  }
  if (!dcd_header(d)) {
    std::fclose(d->f);
    delete d;
    return fail(FZ_ERR_IO, std::string("write error on ") + path);
  }
  *out = d;
  return FZ_OK;
}

extern "C" fz_status fz_dcd_write(fz_dcd* d) {
  if (!d || !d->f) return fail(FZ_ERR_ARG, "null trajectory");
  fz_system* s = d->sys;
  if (!s->eng) return fail(FZ_ERR_STATE, "the system's device state is gone");
  const int n = s->top.n;
  d->pos.resize(3 * (size_t)n);
  d->buf.resize((size_t)n);
  fz_status r;
  if ((r = fz_get_state_f32(s, d->pos.data(), nullptr))) return r;
  const Engine* e = s->eng;
  const double cell[6] = {e->box_d[0], 0.0, e->box_d[1], 0.0, 0.0, e->box_d[2]};
  bool ok = rec(d->f, cell, sizeof cell);
  for (int c = 0; ok && c < 3; ++c) {
    for (int i = 0; i < n; ++i) d->buf[i] = d->pos[3 * (size_t)i + c];
    ok = rec(d->f, d->buf.data(), 4u * (uint32_t)n);
  }
  if (!ok) return fail(FZ_ERR_IO, "trajectory write error");
  d->frames++;
  return FZ_OK;
}

extern "C" fz_status fz_dcd_close(fz_dcd* d) {
  if (!d) return FZ_OK;
  bool ok = true;
  if (d->f) {
    // the header's frame and step counts are those written
    ok = std::fseek(d->f, 0, SEEK_SET) == 0 && dcd_header(d);
    ok = (std::fclose(d->f) == 0) && ok;
  }
  delete d;
  return ok ? FZ_OK : fail(FZ_ERR_IO, "trajectory close error");
}
