// Drop-in check: reference-style user code compiled against the cukd/ shim
// headers and linked to libcukd_b200.so.  Mirrors the reference's own tests
// (testing/testPayloadSampleFromReadme.cu, testing/issue5.cu,
// testing/floatN-knn-and-fcp.cu user kernels, samples/knn-float3-spatialkdtree.cu)
// and dumps its results to <outdir> for tests/test_gpu_shim.py to compare
// with the CPU oracle.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <random>
#include <string>
#include <vector>

#include "cukd/kdtree.h"

struct PointPlusPayload {
  float3 position;
  int payload;
};
struct PointPlusPayload_traits : public cukd::default_data_traits<float3> {
  using data_t = PointPlusPayload;
  static inline __both__ float3 get_point(const data_t &d) { return d.position; }
  static inline __both__ float get_coord(const data_t &d, int dim)
  {
    return cukd::get_coord(d.position, dim);
  }
};

struct PointAndDim {
  float3 point;
  int dim;
};
struct PointAndDim_traits : public cukd::default_data_traits<float3> {
  enum { has_explicit_dim = true };
  using data_t = PointAndDim;
  static inline __both__ const float3 &get_point(const data_t &d) { return d.point; }
  static inline __both__ float get_coord(const data_t &d, int dim)
  {
    return cukd::get_coord(d.point, dim);
  }
  static inline __both__ int get_dim(const data_t &d) { return d.dim; }
  static inline __both__ void set_dim(data_t &d, int dim) { d.dim = dim; }
};

template <typename T> static void dump(const std::string &path, const std::vector<T> &v)
{
  FILE *f = fopen(path.c_str(), "wb");
  fwrite(v.data(), sizeof(T), v.size(), f);
  fclose(f);
}

// 8-dim points, the reference's own vec_float<N> (cukd-math.h:133-181)
using Vec8 = cukd::vec_float<8>;
__global__ void knn8_vec8(const Vec8 *tree, int n, const Vec8 *q, int nq, int *ids)
{
  const int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= nq) return;
  cukd::FixedCandidateList<8> result(INFINITY);
  cukd::stackBased::knn<cukd::FixedCandidateList<8>, Vec8>(result, q[i], tree, n);
  for (int j = 0; j < 8; j++) ids[i * 8 + j] = result.get_pointID(j);
}

__global__ void knn8(const PointPlusPayload *tree, int n, const float3 *q, int nq, int *ids,
                     float *d2)
{
  const int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= nq) return;
  cukd::FixedCandidateList<8> result(INFINITY);
  cukd::stackBased::knn<cukd::FixedCandidateList<8>, PointPlusPayload, PointPlusPayload_traits>(
      result, q[i], tree, n);
  for (int j = 0; j < 8; j++) {
    ids[i * 8 + j] = result.get_pointID(j);
    d2[i * 8 + j] = result.get_dist2(j);
  }
}

__global__ void fcp_cct(const PointAndDim *tree, int n, const cukd::box_t<float3> *bounds,
                        const float3 *q, int nq, int *ids)
{
  const int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= nq) return;
  ids[i] = cukd::cct::fcp<PointAndDim, PointAndDim_traits>(q[i], *bounds, tree, n);
}

__global__ void knn_heap_stackfree(const PointAndDim *tree, int n, const float3 *q, int nq,
                                   int *ids)
{
  const int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= nq) return;
  cukd::HeapCandidateList<20> result(INFINITY);
  cukd::stackFree::knn<cukd::HeapCandidateList<20>, PointAndDim, PointAndDim_traits>(
      result, q[i], tree, n);
  for (int j = 0; j < 20; j++) ids[i * 20 + j] = result.get_pointID(j);
}

__global__ void spatial_knn(cukd::SpatialKDTree<float3> tree, const float3 *q, int nq, int *ids)
{
  const int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= nq) return;
  cukd::HeapCandidateList<16> result(INFINITY);
  cukd::cct::knn(result, tree, q[i]);
  for (int j = 0; j < 16; j++) ids[i * 16 + j] = result.get_pointID(j);
}

__global__ void fcp_issue5(const float3 *tree, int n, float3 q, int *out)
{
  cukd::FcpSearchParams params;
  params.cutOffRadius = 5.f;
  out[0] = cukd::stackBased::fcp(q, tree, n, params);
}

int main(int argc, char **argv)
{
  const std::string out = argc > 1 ? argv[1] : ".";
  const int n = 20000, nq = 5000;
  std::mt19937 gen(1234);
  std::uniform_real_distribution<float> U(0.f, 1.f);
  std::vector<float3> pts(n), qs(nq);
  for (auto &p : pts) p = make_float3(float(int(U(gen) * 50)) / 50.f, U(gen), U(gen));  // ties in x
  for (auto &q : qs) q = make_float3(U(gen), U(gen), U(gen));
  dump(out + "/points.bin", pts);
  dump(out + "/queries.bin", qs);
  float3 *dq;
  CUKD_CUDA_CALL(Malloc(&dq, sizeof(float3) * nq));
  CUKD_CUDA_CALL(Memcpy(dq, qs.data(), sizeof(float3) * nq, cudaMemcpyHostToDevice));

  // 0) point files: cukd::loadPoints reads the count + records layout
  {
    const std::string f = out + "/points_loadpoints.bin";
    std::ofstream o(f, std::ios::binary);
    const uint64_t cnt = uint64_t(n);
    o.write(reinterpret_cast<const char *>(&cnt), sizeof(cnt));
    o.write(reinterpret_cast<const char *>(pts.data()), sizeof(float3) * n);
    o.close();
    int count = 0;
    float3 *lp = cukd::loadPoints<float3>(f, count);
    if (count != n || memcmp(lp, pts.data(), sizeof(float3) * n) != 0)
      throw std::runtime_error("loadPoints returned different records");
    cudaFree(lp);
    std::printf("loadPoints OK\n");
  }

  // 1) README sample: point + payload, default builder, user kNN kernel
  {
    std::vector<PointPlusPayload> data(n);
    for (int i = 0; i < n; i++) data[i] = {pts[i], i};
    PointPlusPayload *d;
    CUKD_CUDA_CALL(Malloc(&d, sizeof(PointPlusPayload) * n));
    CUKD_CUDA_CALL(Memcpy(d, data.data(), sizeof(PointPlusPayload) * n, cudaMemcpyHostToDevice));
    cukd::buildTree<PointPlusPayload, PointPlusPayload_traits>(d, n);
    CUKD_CUDA_CALL(Memcpy(data.data(), d, sizeof(PointPlusPayload) * n, cudaMemcpyDeviceToHost));
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = data[i].payload;
    dump(out + "/payload_order.bin", order);
    int *ids;
    float *d2;
    CUKD_CUDA_CALL(Malloc(&ids, sizeof(int) * nq * 8));
    CUKD_CUDA_CALL(Malloc(&d2, sizeof(float) * nq * 8));
    knn8<<<(nq + 127) / 128, 128>>>(d, n, dq, nq, ids, d2);
    CUKD_CUDA_SYNC_CHECK();
    std::vector<int> hi(nq * 8);
    std::vector<float> hd(nq * 8);
    CUKD_CUDA_CALL(Memcpy(hi.data(), ids, sizeof(int) * nq * 8, cudaMemcpyDeviceToHost));
    CUKD_CUDA_CALL(Memcpy(hd.data(), d2, sizeof(float) * nq * 8, cudaMemcpyDeviceToHost));
    dump(out + "/knn8_ids.bin", hi);
    dump(out + "/knn8_d2.bin", hd);
    cudaFree(ids);
    cudaFree(d2);
    cudaFree(d);
  }
  // 2) explicit split dims (widest extent), inPlace builder name, cct::fcp
  {
    std::vector<PointAndDim> data(n);
    for (int i = 0; i < n; i++) data[i] = {pts[i], -1};
    PointAndDim *d;
    cukd::box_t<float3> *bounds;
    CUKD_CUDA_CALL(Malloc(&d, sizeof(PointAndDim) * n));
    CUKD_CUDA_CALL(MallocManaged(&bounds, sizeof(*bounds)));
    CUKD_CUDA_CALL(Memcpy(d, data.data(), sizeof(PointAndDim) * n, cudaMemcpyHostToDevice));
    bool threw = false;
    try {
      cukd::buildTree_inPlace<PointAndDim, PointAndDim_traits>(d, n);  // no bounds: must throw
    } catch (const std::runtime_error &) {
      threw = true;
    }
    if (!threw) {
      printf("FAIL: explicit dims without world bounds did not throw\n");
      return 1;
    }
    cukd::buildTree_inPlace<PointAndDim, PointAndDim_traits>(d, n, bounds);
    CUKD_CUDA_CALL(Memcpy(data.data(), d, sizeof(PointAndDim) * n, cudaMemcpyDeviceToHost));
    dump(out + "/dim_tree.bin", data);
    int *ids;
    CUKD_CUDA_CALL(Malloc(&ids, sizeof(int) * nq * 20));
    fcp_cct<<<(nq + 127) / 128, 128>>>(d, n, bounds, dq, nq, ids);
    CUKD_CUDA_SYNC_CHECK();
    std::vector<int> hi(nq);
    CUKD_CUDA_CALL(Memcpy(hi.data(), ids, sizeof(int) * nq, cudaMemcpyDeviceToHost));
    dump(out + "/fcp_cct.bin", hi);
    knn_heap_stackfree<<<(nq + 127) / 128, 128>>>(d, n, dq, nq, ids);
    CUKD_CUDA_SYNC_CHECK();
    std::vector<int> hk(nq * 20);
    CUKD_CUDA_CALL(Memcpy(hk.data(), ids, sizeof(int) * nq * 20, cudaMemcpyDeviceToHost));
    dump(out + "/knn20_heap_sf.bin", hk);
    std::vector<float> hb(6);
    for (int dd = 0; dd < 3; dd++) {
      hb[dd] = cukd::get_coord(bounds->lower, dd);
      hb[3 + dd] = cukd::get_coord(bounds->upper, dd);
    }
    dump(out + "/dim_bounds.bin", hb);
    cudaFree(ids);
    cudaFree(d);
    cudaFree(bounds);
  }
  // 3) spatial k-d tree, cct::knn with a heap list
  {
    float3 *d;
    CUKD_CUDA_CALL(Malloc(&d, sizeof(float3) * n));
    CUKD_CUDA_CALL(Memcpy(d, pts.data(), sizeof(float3) * n, cudaMemcpyHostToDevice));
    cukd::SpatialKDTree<float3> tree;
    cukd::buildTree(tree, d, n);
    int *ids;
    CUKD_CUDA_CALL(Malloc(&ids, sizeof(int) * nq * 16));
    spatial_knn<<<(nq + 127) / 128, 128>>>(tree, dq, nq, ids);
    CUKD_CUDA_SYNC_CHECK();
    std::vector<int> hk(nq * 16);
    CUKD_CUDA_CALL(Memcpy(hk.data(), ids, sizeof(int) * nq * 16, cudaMemcpyDeviceToHost));
    dump(out + "/spatial_knn16.bin", hk);
    cukd::free(tree);
    cudaFree(ids);
    cudaFree(d);
  }
  // 4) empty input (testing/testBuilderEmptyInput.cu)
  cukd::buildTree<float3>(nullptr, 0);
  // 5) issue 5 (testing/issue5.cu): 90,167 points, srand(33)/rand() as in
  //    the test's listing (the MSVC LCG), cut-off 5, expected 2.8466301
  {
    const int m = 90167;
    std::vector<float3> p5(m);
    uint32_t x = 33;
    auto rnd = [&]() {
      x = x * 214013u + 2531011u;
      return int((x >> 16) & 0x7fff);
    };
    const double scale = 2.0 * 100.0 / 32767.0;
    for (auto &p : p5) {
      p.x = float(rnd() * scale - 100.0);
      p.y = float(rnd() * scale - 100.0);
      p.z = float(rnd() * scale - 100.0);
    }
    float3 *d;
    int *res;
    CUKD_CUDA_CALL(Malloc(&d, sizeof(float3) * m));
    CUKD_CUDA_CALL(MallocManaged(&res, sizeof(int)));
    CUKD_CUDA_CALL(Memcpy(d, p5.data(), sizeof(float3) * m, cudaMemcpyHostToDevice));
    cukd::buildTree<float3>(d, m);
    const float3 q = make_float3(-98.4496613f, 76.9219055f, 25.8888512f);
    fcp_issue5<<<1, 1>>>(d, m, q, res);
    CUKD_CUDA_SYNC_CHECK();
    float3 pt;
    CUKD_CUDA_CALL(Memcpy(&pt, d + res[0], sizeof(float3), cudaMemcpyDeviceToHost));
    const float dist = cukd::sqrDistance(pt, q);
    printf("issue5: closest %d sqrDist %.7f (expected 2.8466301)\n", res[0], dist);
    if (dist != 2.8466301f) {
      printf("FAIL: issue5\n");
      return 1;
    }
    cudaFree(d);
    cudaFree(res);
  }
  // 6) vec_float<8>: the reference builder test's N = 8 inputs (unique
  //    integer coordinates, scrambled), buildTree and a user kNN kernel
  {
    const int m = 10000, mq = 2000;
    std::vector<int> u(m * 8);
    for (int i = 0; i < m * 8; i++) u[i] = i;
    std::mt19937 g8(88);
    for (int i = m * 8 - 1; i > 0; --i) std::swap(u[i], u[std::uniform_int_distribution<>(0, i)(g8)]);
    std::vector<Vec8> p8(m), q8(mq);
    for (int i = 0; i < m; i++)
      for (int d = 0; d < 8; d++) p8[i].v[d] = float(u[i * 8 + d]);
    std::uniform_real_distribution<float> U8(0.f, float(m * 8));
    for (auto &q : q8)
      for (int d = 0; d < 8; d++) q.v[d] = U8(g8);
    dump(out + "/vec8_points.bin", p8);
    dump(out + "/vec8_queries.bin", q8);
    Vec8 *d, *dq;
    int *ids;
    CUKD_CUDA_CALL(Malloc(&d, sizeof(Vec8) * m));
    CUKD_CUDA_CALL(Malloc(&dq, sizeof(Vec8) * mq));
    CUKD_CUDA_CALL(Malloc(&ids, sizeof(int) * mq * 8));
    CUKD_CUDA_CALL(Memcpy(d, p8.data(), sizeof(Vec8) * m, cudaMemcpyHostToDevice));
    CUKD_CUDA_CALL(Memcpy(dq, q8.data(), sizeof(Vec8) * mq, cudaMemcpyHostToDevice));
    cukd::buildTree<Vec8>(d, m);
    knn8_vec8<<<(mq + 127) / 128, 128>>>(d, m, dq, mq, ids);
    CUKD_CUDA_SYNC_CHECK();
    CUKD_CUDA_CALL(Memcpy(p8.data(), d, sizeof(Vec8) * m, cudaMemcpyDeviceToHost));
    std::vector<int> hi(mq * 8);
    CUKD_CUDA_CALL(Memcpy(hi.data(), ids, sizeof(int) * mq * 8, cudaMemcpyDeviceToHost));
    dump(out + "/vec8_tree.bin", p8);
    dump(out + "/vec8_knn8.bin", hi);
    cudaFree(d);
    cudaFree(dq);
    cudaFree(ids);
  }
  printf("shim_test OK\n");
  return 0;
}
