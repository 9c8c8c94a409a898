// The reference's files, byte-compatible, through the public entry points:
//  - suspend_job / continue_job (PIC/3d_pic458_domain.c:7629-7911):
//    suspend-<rank>-field.dat (the Grid records, :115-123, for every node,
//    z fastest) and suspend-<rank>-<thread>-{ion,electron}.dat (the Particle
//    structs, :134-141: x y z vx vy vz n, int flag, the two list links);
//  - output (:4834-4883): fdtd458-<rx>-<ry>-<step>.dat, 23 columns per
//    interior node;
//  - the lines thrust_f and thrust_fave append to thrust458.txt (:5111-5119)
//    and thrust458_ave.txt (:5266-5276).
// Included at the end of api.cu (host code only).

#include <cerrno>
#include <string>

namespace {

constexpr int kVersion = 458;  // the reference's `version` (:50), part of its file names

// The Particle struct as the reference writes it with fwrite (x86-64 layout).
struct FileParticle {
  double x, y, z, vx, vy, vz, n;
  int flag;
  int pad;
  unsigned long long prev, next;
};
static_assert(sizeof(FileParticle) == 80, "reference Particle record is 80 bytes");

std::string join(const char* dir, const std::string& name) {
  std::string d = (dir && *dir) ? dir : ".";
  if (d.back() != '/') d += '/';
  return d + name;
}

long long grid_nodes(const pic_ctx* c) { return (long long)c->g.gx * c->g.gy * c->g.gz; }

}  // namespace

extern "C" {

int pic_save_checkpoint(pic_ctx* c, const char* dir, int rank, int nthreads) {
  CKR(check_ctx(c));
  if (nthreads < 1 || rank < 0) return PIC_ERR_ARG;
  const long long nodes = grid_nodes(c);
  std::vector<double> rec((size_t)nodes * PIC_GRID_RECORD);
  CKR(pic_get_grid(c, rec.data()));
  {
    const std::string f = join(dir, "suspend-" + std::to_string(rank) + "-field.dat");
    FILE* fp = fopen(f.c_str(), "wb");
    if (!fp) return PIC_ERR_ARG;
    const size_t w = fwrite(rec.data(), sizeof(double) * PIC_GRID_RECORD, (size_t)nodes, fp);
    fclose(fp);
    if (w != (size_t)nodes) return PIC_ERR_ARG;
  }
  const char* names[2] = {"ion", "electron"};
  for (int s = 0; s < 2; ++s) {
    long long n = 0;
    CKR(pic_particle_count(c, s, &n));
    std::vector<double> rows((size_t)std::max(n, 1LL) * PIC_PARTICLE_ROW);
    long long got = 0;
    CKR(pic_get_particles(c, s, rows.data(), nullptr, n, &got));
    for (int t = 0; t < nthreads; ++t) {
      const long long a = got * t / nthreads, b = got * (t + 1) / nthreads;
      const std::string f =
          join(dir, "suspend-" + std::to_string(rank) + "-" + std::to_string(t) + "-" + names[s] + ".dat");
      FILE* fp = fopen(f.c_str(), "wb");
      if (!fp) return PIC_ERR_ARG;
      std::vector<FileParticle> buf;
      buf.reserve(65536);
      bool ok = true;
      for (long long i = a; i < b; ++i) {
        const double* r = rows.data() + PIC_PARTICLE_ROW * i;
        FileParticle p{r[0], r[1], r[2], r[3], r[4], r[5], r[6], 1, 0, 0ull, 0ull};
        buf.push_back(p);
        if (buf.size() == 65536 || i == b - 1) {
          ok = ok && fwrite(buf.data(), sizeof(FileParticle), buf.size(), fp) == buf.size();
          buf.clear();
        }
      }
      fclose(fp);
      if (!ok) return PIC_ERR_ARG;
    }
  }
  return PIC_OK;
}

int pic_load_checkpoint(pic_ctx* c, const char* dir, int rank, int nthreads) {
  CKR(check_ctx(c));
  if (nthreads < 1 || rank < 0) return PIC_ERR_ARG;
  const long long nodes = grid_nodes(c);
  std::vector<double> rec((size_t)nodes * PIC_GRID_RECORD);
  {
    const std::string f = join(dir, "suspend-" + std::to_string(rank) + "-field.dat");
    FILE* fp = fopen(f.c_str(), "rb");
    if (!fp) return PIC_ERR_ARG;
    const size_t r = fread(rec.data(), sizeof(double) * PIC_GRID_RECORD, (size_t)nodes, fp);
    const bool extra = fgetc(fp) != EOF;  // a field file of another grid size
    fclose(fp);
    if (r != (size_t)nodes || extra) return PIC_ERR_ARG;
  }
  const char* names[2] = {"ion", "electron"};
  std::vector<double> rows[2];
  for (int s = 0; s < 2; ++s) {
    for (int t = 0; t < nthreads; ++t) {
      const std::string f =
          join(dir, "suspend-" + std::to_string(rank) + "-" + std::to_string(t) + "-" + names[s] + ".dat");
      FILE* fp = fopen(f.c_str(), "rb");
      if (!fp) return PIC_ERR_ARG;
      // a file cut inside a record is rejected before anything is loaded
      if (fseek(fp, 0, SEEK_END) != 0 || ftell(fp) < 0 || ftell(fp) % (long)sizeof(FileParticle) != 0 ||
          fseek(fp, 0, SEEK_SET) != 0) {
        fclose(fp);
        return PIC_ERR_ARG;
      }
      FileParticle p;
      while (fread(&p, sizeof(p), 1, fp) == 1) {
        const double r[PIC_PARTICLE_ROW] = {p.x, p.y, p.z, p.vx, p.vy, p.vz, p.n};
        rows[s].insert(rows[s].end(), r, r + PIC_PARTICLE_ROW);
        if (p.flag != 1) {
          fclose(fp);
          return PIC_ERR_ARG;  // this path keeps flag = 1 for every particle
        }
      }
      fclose(fp);
    }
  }
  CKR(pic_set_grid(c, rec.data()));
  for (int s = 0; s < 2; ++s) {
    const long long n = (long long)rows[s].size() / PIC_PARTICLE_ROW;
    CKR(pic_set_particles(c, s, n ? rows[s].data() : nullptr, nullptr, n));
  }
  // continue_job seeds the random streams afresh (:7770-7777)
  long long zero_p = 0, zero_v = 0;
  CKR(pic_rng_counters(c, &zero_p, &zero_v, 1));
  return PIC_OK;
}

int pic_write_output(pic_ctx* c, const char* dir, int step) {
  CKR(check_ctx(c));
  const Geom& g = c->g;
  std::vector<double> rec((size_t)grid_nodes(c) * PIC_GRID_RECORD);
  CKR(pic_get_grid(c, rec.data()));
  const std::string f = join(dir, "fdtd" + std::to_string(kVersion) + "-0-0-" + std::to_string(step) + ".dat");
  FILE* fp = fopen(f.c_str(), "w");
  if (!fp) return PIC_ERR_ARG;
  enum { BX, BY, BZ, B0X, B0Y, B0Z, EX, EY, EZ, JIX, JIY, JIZ, JEX, JEY, JEZ, NI, NE, PHI };
  auto G = [&](int k, int l, int m, int f) { return rec[(((size_t)k * g.gy + l) * g.gz + m) * PIC_GRID_RECORD + f]; };
  const double dx = c->cfg.dx;
  const int Nx = g.nx, Ny = g.ny, Nz = g.nz;
  bool ok = true;
  for (int k = 2; k < Nx + 2 && ok; k++)
    for (int l = 2; l < Ny + 2 && ok; l++)
      for (int m = 2; m < Nz + 2; m++) {
        const double bxa = (G(k, l, m, BX) + G(k, l + 1, m, BX) + G(k, l, m + 1, BX) + G(k, l + 1, m + 1, BX)) / 4.;
        const double bya = (G(k, l, m, BY) + G(k + 1, l, m, BY) + G(k, l, m + 1, BY) + G(k + 1, l, m + 1, BY)) / 4.;
        const double bza = (G(k, l, m, BZ) + G(k + 1, l, m, BZ) + G(k, l + 1, m, BZ) + G(k + 1, l + 1, m, BZ)) / 4.;
        const double b0xa =
            (G(k, l, m, B0X) + G(k, l + 1, m, B0X) + G(k, l, m + 1, B0X) + G(k, l + 1, m + 1, B0X)) / 4.;
        const double b0ya =
            (G(k, l, m, B0Y) + G(k + 1, l, m, B0Y) + G(k, l, m + 1, B0Y) + G(k + 1, l, m + 1, B0Y)) / 4.;
        const double b0za =
            (G(k, l, m, B0Z) + G(k + 1, l, m, B0Z) + G(k, l + 1, m, B0Z) + G(k + 1, l + 1, m, B0Z)) / 4.;
        const int rc = fprintf(
            fp,
            "%.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E %.3E "
            "%.3E %.3E %.3E\n",
            (k - 2 - 1 * Nx / 2) * dx, (l - 2 - 1 * Ny / 2) * dx, (m - (Nz + 4) / 2) * dx, G(k, l, m, NI),
            G(k, l, m, NE), G(k, l, m, NI) - G(k, l, m, NE), (G(k + 1, l, m, EX) + G(k, l, m, EX)) / 2.,
            (G(k, l + 1, m, EY) + G(k, l, m, EY)) / 2., (G(k, l, m + 1, EZ) + G(k, l, m, EZ)) / 2., bxa, bya, bza,
            G(k, l, m, JIX), G(k, l, m, JIY), G(k, l, m, JIZ), G(k, l, m, JEX), G(k, l, m, JEY), G(k, l, m, JEZ),
            G(k, l, m, PHI), sqrt(pow(bxa, 2) + pow(bya, 2) + pow(bza, 2)), bxa - b0xa, bya - b0ya, bza - b0za);
        if (rc < 0) {
          ok = false;
          break;
        }
      }
  fclose(fp);
  return ok ? PIC_OK : PIC_ERR_ARG;
}

int pic_append_thrust(pic_ctx* c, const char* dir, int step) {
  double F[PIC_NUM_THRUST], E[PIC_NUM_ENERGY];
  CKR(pic_thrust_f(c, F, E));
  const std::string f = join(dir, "thrust" + std::to_string(kVersion) + ".txt");
  FILE* fp = fopen(f.c_str(), "a");
  if (!fp) return PIC_ERR_ARG;
  int rc = fprintf(fp, "%d", step);
  for (int q = 0; q < PIC_NUM_THRUST && rc >= 0; ++q) rc = fprintf(fp, " %.3E", F[q]);
  for (int q = 0; q < PIC_NUM_ENERGY && rc >= 0; ++q) rc = fprintf(fp, " %.8E", E[q]);
  if (rc >= 0) rc = fprintf(fp, "\n");
  fclose(fp);
  return rc < 0 ? PIC_ERR_ARG : PIC_OK;
}

int pic_append_thrust_ave(pic_ctx* c, const char* dir, int step) {
  CKR(check_ctx(c));
  if (step % 500 != 0) return PIC_OK;  // thrust_fave writes every 500 steps (:5267)
  double Fave[PIC_NUM_THRUST];
  CKR(pic_thrust_fave(c, Fave, 1));
  const std::string f = join(dir, "thrust" + std::to_string(kVersion) + "_ave.txt");
  FILE* fp = fopen(f.c_str(), "a");
  if (!fp) return PIC_ERR_ARG;
  int rc = fprintf(fp, "%d", step);
  for (int q = 0; q < PIC_NUM_THRUST && rc >= 0; ++q) rc = fprintf(fp, " %.3E", Fave[q]);
  if (rc >= 0) rc = fprintf(fp, "\n");
  fclose(fp);
  return rc < 0 ? PIC_ERR_ARG : PIC_OK;
}

}  // extern "C"
