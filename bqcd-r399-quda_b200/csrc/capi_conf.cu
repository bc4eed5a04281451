// capi_conf.cu -- C ABI of BQCD's configuration files (include/bqcdg.h):
// the host side of conf_write / conf_read; the reordering, byte swap and
// check sums run in confio.cu.
#include "ctx.cuh"

using namespace bqcdg;
using namespace bqcdg_host;

// ---------------------------------------------------------------------------
// configuration files (conf.F90:219-470, conf_info.F90, cksum.c)
// ---------------------------------------------------------------------------
namespace {

// cksum's end: the byte count fed in least significant byte first, then the
// complement (cksum.c:150-165), applied to the raw register of the data
unsigned cksum_finish(unsigned crc, unsigned long long nbytes) {
  static unsigned tab[256];
  static bool ready = false;
  if (!ready) {
    for (unsigned b = 0; b < 256; b++) {
      unsigned r = b << 24;
      for (int k = 0; k < 8; k++) r = (r & 0x80000000u) ? (r << 1) ^ 0x04C11DB7u : (r << 1);
      tab[b] = r;
    }
    ready = true;
  }
  for (unsigned long long n = nbytes; n > 0; n >>= 8) crc = (crc << 8) ^ tab[((crc >> 24) ^ (unsigned)(n & 0xFF))];
  return ~crc;
}

std::string slice_file(const std::string& base, int t) {
  char buf[32];
  std::snprintf(buf, sizeof(buf), ".%02d.u", t);
  return base + buf;
}

std::string file_part(const std::string& path) {
  const size_t k = path.rfind('/');
  return k == std::string::npos ? path : path.substr(k + 1);
}

std::string dir_part(const std::string& path) {
  const size_t k = path.rfind('/');
  return k == std::string::npos ? std::string() : path.substr(0, k + 1);
}

// pinned host buffer of one slice, released on scope exit
struct PinnedSlice {
  void* p = nullptr;
  ~PinnedSlice() {
    if (p) cudaFreeHost(p);
  }
};

}  // namespace

extern "C" {

int bqcdg_conf_write(bqcdg_ctx* c, const char* base, bqcdg_conf_meta* meta) {
  if (!c || !base || !meta) return BQCDG_EINVAL;
  if (!c->have_gauge) return BQCDG_ENOGAUGE;
  CK(cudaSetDevice(c->device));
  const Geom& g = c->g;
  const size_t nbytes = (size_t)g.L[0] * g.L[1] * g.L[2] * 384;
  CK(c->stage(nbytes));
  PinnedSlice host;
  CK(cudaMallocHost(&host.p, nbytes));
  double sg;
  int st = bqcdg_sg(c, &sg);
  if (st) return st;
  meta->plaq_energy = sg / (6.0 * 2.0 * g.volh);
  for (int d = 0; d < 4; d++) {
    meta->L[d] = g.L[d];
    meta->bc[d] = g.bcsign[d];
  }
  unsigned* acc = reinterpret_cast<unsigned*>(c->dres);
  std::vector<unsigned> sums(g.L[3]);
  for (int t = 0; t < g.L[3]; t++) {
    CK(cudaMemsetAsync(acc, 0, sizeof(unsigned), c->stream));
    CK(launch_links_to_file(g, c->gauge64, t, c->staging, acc, c->stream));
    CK(cudaMemcpyAsync(host.p, c->staging, nbytes, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(c->hres, acc, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    sums[t] = cksum_finish(*reinterpret_cast<unsigned*>(c->hres), nbytes);
    FILE* f = std::fopen(slice_file(base, t).c_str(), "wb");
    if (!f) return BQCDG_EIO;
    const size_t w = std::fwrite(host.p, 1, nbytes, f);
    if (std::fclose(f) != 0 || w != nbytes) return BQCDG_EIO;
  }
  FILE* f = std::fopen((std::string(base) + ".info").c_str(), "w");
  if (!f) return BQCDG_EIO;
  char host_name[64] = "unknown", date[32] = "-", clock[32] = "-";
  gethostname(host_name, sizeof(host_name) - 1);
  const std::time_t now = std::time(nullptr);
  std::strftime(date, sizeof(date), "%Y-%m-%d", std::localtime(&now));
  std::strftime(clock, sizeof(clock), "%H:%M:%S", std::localtime(&now));
  // the ConfInfoHeader block of write_conf_info_header (conf_info.F90:28-63)
  std::fprintf(f, " >BeginConfInfoHeader\n Format 3\n Program bqcd-b200 1\n Run %d\n Traj %d\n Host %s\n Date %s %s\n",
               meta->run, meta->traj, host_name, date, clock);
  std::fprintf(f, " L%3d%3d%3d%3d\n bc_fermions%3d%3d%3d%3d\n REAL_kind 8\n PlaqEnergy %25.14E\n", g.L[0], g.L[1],
               g.L[2], g.L[3], g.bcsign[0], g.bcsign[1], g.bcsign[2], g.bcsign[3], meta->plaq_energy);
  static const char* const pre[2] = {"", "former_"};
  for (int k = 0; k < 2; k++) {
    std::fprintf(f, " %sensemble %d\n", pre[k], meta->ensemble[k]);
    std::fprintf(f, " %sbeta %.17g\n %skappa %.17g\n %scsw %.17g\n %scsw_kappa %.17g\n %sh %.17g\n", pre[k],
                 meta->beta[k], pre[k], meta->kappa[k], pre[k], meta->csw[k], pre[k], meta->csw_kappa[k], pre[k],
                 meta->h[k]);
  }
  std::fprintf(f, " >EndConfInfoHeader\n >BeginCheckSum\n");
  for (int t = 0; t < g.L[3]; t++)
    std::fprintf(f, " %s %u %zu\n", file_part(slice_file(base, t)).c_str(), sums[t], nbytes);
  std::fprintf(f, " >EndCheckSum\n");
  if (std::fclose(f) != 0) return BQCDG_EIO;
  return BQCDG_OK;
}

int bqcdg_conf_read(bqcdg_ctx* c, const char* info_file, bqcdg_conf_meta* meta) {
  if (!c || !info_file || !meta) return BQCDG_EINVAL;
  std::memset(meta, 0, sizeof(*meta));
  FILE* f = std::fopen(info_file, "r");
  if (!f) return BQCDG_EIO;
  // keyword lines of the header (read_keyword_*, conf_info.F90:65-90) and
  // the CheckSum block (read_cksum, conf_info.F90:140-160)
  std::map<std::string, std::string> keys;
  std::vector<std::pair<std::string, unsigned long long>> files;
  char line[1024];
  int block = 0;  // 1 header, 2 check sums
  while (std::fgets(line, sizeof(line), f)) {
    char w0[512] = "", rest[512] = "";
    if (std::sscanf(line, " %511s %511[^\n]", w0, rest) < 1) continue;
    const std::string k(w0);
    if (k == ">BeginConfInfoHeader") block = 1;
    else if (k == ">BeginCheckSum") block = 2;
    else if (k.rfind(">End", 0) == 0) block = 0;
    else if (block == 1) keys[k] = rest;
    else if (block == 2) {
      unsigned long long sum = 0;
      if (std::sscanf(rest, "%llu", &sum) != 1) {
        std::fclose(f);
        return BQCDG_EIO;
      }
      files.emplace_back(k, sum);
    }
  }
  std::fclose(f);
  auto geti = [&](const char* k, int* v, int n) {
    auto it = keys.find(k);
    if (it == keys.end()) return false;
    const char* p = it->second.c_str();
    for (int j = 0; j < n; j++) {
      int used = 0;
      if (std::sscanf(p, "%d%n", &v[j], &used) != 1) return false;
      p += used;
    }
    return true;
  };
  auto getd = [&](const char* k, double* v) {
    auto it = keys.find(k);
    return it != keys.end() && std::sscanf(it->second.c_str(), "%lf", v) == 1;
  };
  int format = 0, rkind = 0;
  if (!geti("Format", &format, 1) || format != 3) return BQCDG_EIO;  // conf_info_version (module_bqcd.F90:38)
  if (!geti("L", meta->L, 4) || !geti("bc_fermions", meta->bc, 4) || !geti("REAL_kind", &rkind, 1) || rkind != 8)
    return BQCDG_EIO;
  geti("Run", &meta->run, 1);
  geti("Traj", &meta->traj, 1);
  getd("PlaqEnergy", &meta->plaq_energy);
  static const char* const pre[2] = {"", "former_"};
  for (int k = 0; k < 2; k++) {
    const std::string p(pre[k]);
    geti((p + "ensemble").c_str(), &meta->ensemble[k], 1);
    getd((p + "beta").c_str(), &meta->beta[k]);
    getd((p + "kappa").c_str(), &meta->kappa[k]);
    getd((p + "csw").c_str(), &meta->csw[k]);
    getd((p + "csw_kappa").c_str(), &meta->csw_kappa[k]);
    getd((p + "h").c_str(), &meta->h[k]);
  }
  const Geom& g = c->g;
  for (int d = 0; d < 4; d++)
    if (meta->L[d] != g.L[d]) return BQCDG_EINVAL;  // check_conf_info_header (conf_info.F90:96-101)
  if ((int)files.size() != g.L[3]) return BQCDG_EIO;
  CK(cudaSetDevice(c->device));
  if (!c->gauge64) CK(c->alloc((void**)&c->gauge64, (size_t)8 * 9 * g.stride * sizeof(double2)));
  const size_t nbytes = (size_t)g.L[0] * g.L[1] * g.L[2] * 384;
  CK(c->stage(nbytes));
  PinnedSlice host;
  CK(cudaMallocHost(&host.p, nbytes));
  // the links are overwritten slice by slice: until all check out, none is loaded
  c->have_gauge = false;
  for (int k = 0; k < 3; k++) c->gauge_s_ok[k] = false;
  c->gauge64r_ok = false;
  const std::string dir = dir_part(info_file);
  unsigned* acc = reinterpret_cast<unsigned*>(c->dres);
  for (int t = 0; t < g.L[3]; t++) {
    const std::string name = files[t].first[0] == '/' ? files[t].first : dir + files[t].first;
    FILE* s = std::fopen(name.c_str(), "rb");
    if (!s) return BQCDG_EIO;
    const size_t r = std::fread(host.p, 1, nbytes, s);
    const bool extra = std::fgetc(s) != EOF;
    std::fclose(s);
    if (r != nbytes || extra) return BQCDG_EIO;
    CK(cudaMemcpyAsync(c->staging, host.p, nbytes, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(acc, 0, sizeof(unsigned), c->stream));
    CK(launch_links_from_file(g, c->staging, t, c->gauge64, acc, c->stream));
    CK(cudaMemcpyAsync(c->hres, acc, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (cksum_finish(*reinterpret_cast<unsigned*>(c->hres), nbytes) != files[t].second) return BQCDG_ECHECKSUM;
  }
  launch_gauge_check(g, c->gauge64, c->red, c->dres, c->stream);
  CKL();
  CK(cudaMemcpyAsync(c->hres, c->dres, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  c->gauge_su3 = c->hres[0] < 1e-10 && c->hres[1] < 1e-10;
  c->have_gauge = true;
  return BQCDG_OK;
}

}  // extern "C"
