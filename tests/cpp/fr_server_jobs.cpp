// A C++ client of the serving C-ABI (include/umpalumpa_fr_server.h), as a host application
// would write it: three reconstruction jobs of different box sizes are opened on one server,
// three client threads stream their projection batches (host memory: half-planes plus 3x3
// rotations) while the server's request loop inserts them, and each finished volume is read
// back.  The same batches then go through the single-job entry points (fr_create / fr_init /
// fr_execute with traverse spaces from fr_compute_traverse_spaces), and the program checks that
// every job's volume and weights agree within relative L2 1e-5.  Prints one line per job and
// exits 0 on success.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <random>
#include <thread>
#include <vector>

#include "umpalumpa_fr.h"
#include "umpalumpa_fr_server.h"

namespace {

struct Job {
  int box = 0, n = 0, batch = 0;
  std::vector<float> fft;  // n x box x (box/2+1) interleaved complex
  std::vector<float> rot;  // n x 9, row-major
  std::vector<float> vol, w, pv, pw;
};

Job make_job(int box, int n, int batch, unsigned seed)
{
  Job J;
  J.box = box;
  J.n = n;
  J.batch = batch;
  std::mt19937 rng(seed);
  std::normal_distribution<float> g(0.f, 1.f);
  const size_t plane = size_t(box) * (box / 2 + 1) * 2;
  J.fft.resize(plane * n);
  for (auto &v : J.fft) v = g(rng) / float(box);
  J.rot.resize(size_t(n) * 9);
  for (int i = 0; i < n; ++i) {  // rotation from a uniform unit quaternion
    float q[4];
    float s = 0.f;
    for (float &c : q) {
      c = g(rng);
      s += c * c;
    }
    s = 1.f / std::sqrt(s);
    const float a = q[0] * s, b = q[1] * s, c = q[2] * s, d = q[3] * s;
    const float m[9] = { a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c),
                         2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b),
                         2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d };
    std::copy(m, m + 9, J.rot.begin() + size_t(i) * 9);
  }
  return J;
}

double rel_l2(const std::vector<float> &a, const std::vector<float> &b)
{
  double num = 0, den = 0;
  for (size_t i = 0; i < a.size(); ++i) {
    num += double(a[i] - b[i]) * (a[i] - b[i]);
    den += double(b[i]) * b[i];
  }
  return den > 0 ? std::sqrt(num / den) : std::sqrt(num);
}

#define CHECK(call)                                                                                   \
  do {                                                                                                \
    const int rc_ = (call);                                                                           \
    if (rc_ != 0) {                                                                                   \
      std::printf("FAIL %s -> %d: %s\n", #call, rc_, fr_last_error());                                \
      return 1;                                                                                       \
    }                                                                                                 \
  } while (0)

#define CUDA(call)                                                                                    \
  do {                                                                                                \
    const cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess) {                                                                          \
      std::printf("FAIL %s: %s\n", #call, cudaGetErrorString(e_));                                   \
      return 1;                                                                                       \
    }                                                                                                 \
  } while (0)

fr_settings settings()
{
  fr_settings s;
  fr_settings_default(&s);
  s.type = FR_TYPE_PRECISE;
  s.interpolation = FR_INTERPOLATION_LOOKUP;
  return s;
}

// The single-job path, one fr_execute per batch.
int run_plain(Job &J, const float *table)
{
  const int v = J.box + 1, X = J.box / 2 + 1;
  const size_t voxels = size_t(v) * v * v;
  fr_handle *h = nullptr;
  CHECK(fr_create(0, nullptr, &h));
  fr_dims d{};
  d.fft_x = X;
  d.fft_y = J.box;
  d.n_projections = J.batch;
  d.volume_x = d.volume_y = d.volume_z = v;
  d.n_spaces = J.batch;
  d.table_elems = 10000;
  const fr_settings s = settings();
  CHECK(fr_init(h, &d, &s));
  void *vol = nullptr;
  float *w = nullptr, *rot = nullptr;
  fr_traverse_space *sp = nullptr;
  CUDA(cudaMalloc(&vol, voxels * 8));
  CUDA(cudaMalloc(reinterpret_cast<void **>(&w), voxels * 4));
  CUDA(cudaMalloc(reinterpret_cast<void **>(&rot), size_t(J.batch) * 9 * sizeof(float)));
  CUDA(cudaMalloc(reinterpret_cast<void **>(&sp), size_t(J.batch) * sizeof(fr_traverse_space)));
  CUDA(cudaMemset(vol, 0, voxels * 8));
  CUDA(cudaMemset(w, 0, voxels * 4));
  const size_t plane = size_t(J.box) * X * 2;
  for (int b0 = 0; b0 < J.n; b0 += J.batch) {
    const int nb = std::min(J.batch, J.n - b0);
    CUDA(cudaMemcpy(rot, J.rot.data() + size_t(b0) * 9, size_t(nb) * 9 * sizeof(float), cudaMemcpyHostToDevice));
    CHECK(fr_compute_traverse_spaces(rot, nb, J.box / 2, J.box, J.box, J.box, 0, s.blob_radius, 1.f, 0, sp, nullptr));
    CHECK(fr_execute(h, J.fft.data() + plane * b0, nullptr, nb, vol, w, sp, nb, table));  // host half-planes
    CHECK(fr_synchronize(h));
  }
  J.pv.resize(voxels * 2);
  J.pw.resize(voxels);
  CUDA(cudaMemcpy(J.pv.data(), vol, voxels * 8, cudaMemcpyDeviceToHost));
  CUDA(cudaMemcpy(J.pw.data(), w, voxels * 4, cudaMemcpyDeviceToHost));
  cudaFree(vol);
  cudaFree(w);
  cudaFree(rot);
  cudaFree(sp);
  fr_destroy(h);
  return 0;
}

}// namespace

int main()
{
  std::vector<Job> jobs = { make_job(32, 300, 70, 1), make_job(48, 500, 120, 2), make_job(64, 400, 90, 3) };
  const fr_settings s = settings();
  fr_server_config cfg;
  fr_server_config_default(&cfg);
  cfg.hbm_budget = 4ull << 30;
  fr_server *srv = nullptr;
  CHECK(fr_server_create(0, &cfg, &s, &srv));
  std::vector<uint64_t> ids(jobs.size());
  for (size_t k = 0; k < jobs.size(); ++k) {
    fr_server_job_desc d{};
    d.fft_x = jobs[k].box / 2 + 1;
    d.fft_y = jobs[k].box;
    d.volume_x = d.volume_y = d.volume_z = jobs[k].box + 1;
    d.image_x = jobs[k].box / 2;
    d.image_y = jobs[k].box;
    d.space_weight = 1.f;
    CHECK(fr_server_open_job(srv, &d, &ids[k]));
  }
  // one client thread per job streams its batches; the buffers are the job's own host arrays,
  // which outlive the job
  std::vector<int> client_rc(jobs.size(), 0);
  std::vector<std::thread> clients;
  for (size_t k = 0; k < jobs.size(); ++k)
    clients.emplace_back([&, k] {
      const Job &J = jobs[k];
      const size_t plane = size_t(J.box) * (J.box / 2 + 1) * 2;
      for (int b0 = 0; b0 < J.n && client_rc[k] == 0; b0 += J.batch) {
        fr_server_batch b{};
        b.fft = J.fft.data() + plane * b0;
        b.rotations = J.rot.data() + size_t(b0) * 9;
        b.n_projections = uint64_t(std::min(J.batch, J.n - b0));
        client_rc[k] = fr_server_submit(srv, ids[k], &b);
        std::this_thread::sleep_for(std::chrono::milliseconds(2 + int(k)));
      }
      if (client_rc[k] == 0) client_rc[k] = fr_server_close_job(srv, ids[k]);
    });
  for (auto &t : clients) t.join();
  for (size_t k = 0; k < jobs.size(); ++k)
    if (client_rc[k] != 0) {
      std::printf("FAIL client %zu: %d %s\n", k, client_rc[k], fr_last_error());
      return 1;
    }
  for (size_t k = 0; k < jobs.size(); ++k) {
    Job &J = jobs[k];
    fr_server_job_info info;
    CHECK(fr_server_wait_job(srv, ids[k], 120.0, &info));
    const size_t voxels = size_t(J.box + 1) * (J.box + 1) * (J.box + 1);
    J.vol.resize(voxels * 2);
    J.w.resize(voxels);
    CHECK(fr_server_read_job(srv, ids[k], J.vol.data(), J.w.data()));
    CHECK(fr_server_release_job(srv, ids[k]));
  }
  fr_server_stats st;
  CHECK(fr_server_get_stats(srv, &st));
  CHECK(fr_server_destroy(srv));

  float *table = nullptr;
  CUDA(cudaMalloc(reinterpret_cast<void **>(&table), 10000 * sizeof(float)));
  CHECK(fr_fill_blob_table(table, 10000, &s, nullptr));
  CUDA(cudaDeviceSynchronize());
  int bad = 0;
  for (auto &J : jobs) {
    if (run_plain(J, table)) return 1;
    const double ev = rel_l2(J.vol, J.pv), ew = rel_l2(J.w, J.pw);
    const bool ok = ev <= 1e-5 && ew <= 1e-5 && rel_l2(J.pw, std::vector<float>(J.pw.size(), 0.f)) > 0;
    std::printf("%s job box %d projections %d: relL2 served vs single-job volume %.2e weights %.2e\n",
      ok ? "PASS" : "FAIL", J.box, J.n, ev, ew);
    bad += !ok;
  }
  cudaFree(table);
  std::printf("server steps %llu, spaces %llu, jobs done %llu\n", (unsigned long long)st.steps,
    (unsigned long long)st.spaces, (unsigned long long)st.jobs_done);
  return bad || st.jobs_done != jobs.size() ? 1 : 0;
}
