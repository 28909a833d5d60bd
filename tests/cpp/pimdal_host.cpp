// pimdal_host.cpp -- a compiled C++ host program on the C ABI of
// include/pimdal_gpu.h: the drop-in for the reference's host programs.
//
// The reference's host programs (e.g. pimdal/main/select/host/
// host_select_sync.cpp:40-89) populate the DPUs' MRAM (populate_mram:
// dpu_broadcast_to + dist_table), launch the DPU kernel (dpu_launch) and
// gather the results (get_results: get_vec of the counts, get_buf of the
// rows).  Here the same three steps are populate (cudaMalloc + pimdal_ingest
// of the host columns), launch (one pimdal_* call on a stream) and
// get_results (the count, pimdal_ctx_sync_status, the rows copied back).
//
//   pimdal_host <dir> select <lo> <hi>  reads sel_keys.i32, writes sel_vals.i32, sel_rows.u32
//   pimdal_host <dir> sort              reads sort_keys.u32, writes sort_keys_out.u32, sort_rows.u32
//   pimdal_host <dir> hash_join         reads hj_bk.i32 hj_bp.i32 hj_pk.i32, writes hj_pay.u32 hj_row.u32
//   pimdal_host <dir> group_by          reads gb_k.i32 gb_v.i64, writes gb_{key,sum,count,min,max}
//
// Files are raw little-endian arrays.  Exit status 0 on success; a library
// status code is printed with pimdal_status_string and returned otherwise.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "pimdal_gpu.h"

namespace {

struct Failure {
  int status;
  std::string where;
};

void check(int status, const char *where) {
  if (status != PIMDAL_OK) throw Failure{status, where};
}
void check_cuda(cudaError_t e, const char *where) {
  if (e != cudaSuccess) throw Failure{PIMDAL_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e)};
}

template <class T>
std::vector<T> read_file(const std::string &path) {
  std::ifstream f(path, std::ios::binary | std::ios::ate);
  if (!f) throw Failure{PIMDAL_ERR_ARG, "cannot read " + path};
  const std::streamsize bytes = f.tellg();
  f.seekg(0);
  std::vector<T> v(bytes / sizeof(T));
  if (bytes) f.read(reinterpret_cast<char *>(v.data()), bytes);
  return v;
}

template <class T>
void write_file(const std::string &path, const T *data, size_t n) {
  std::ofstream f(path, std::ios::binary);
  if (n) f.write(reinterpret_cast<const char *>(data), sizeof(T) * n);
  if (!f) throw Failure{PIMDAL_ERR_ARG, "cannot write " + path};
}

// One device session: a context, a stream and the device buffers it made.
struct Session {
  pimdal_ctx_t *ctx = nullptr;
  cudaStream_t s = nullptr;
  std::vector<void *> owned;

  Session() {
    check(pimdal_ctx_create(&ctx, 0), "pimdal_ctx_create");
    check_cuda(cudaStreamCreate(&s), "cudaStreamCreate");
  }
  ~Session() {
    cudaStreamSynchronize(s);
    for (void *p : owned) cudaFree(p);
    cudaStreamDestroy(s);
    pimdal_ctx_destroy(ctx);
  }
  template <class T>
  T *alloc(size_t n) {
    void *p = nullptr;
    check_cuda(cudaMalloc(&p, sizeof(T) * (n ? n : 1)), "cudaMalloc");
    owned.push_back(p);
    return static_cast<T *>(p);
  }
  // populate: a host column into a new device buffer (the dist_table step)
  template <class T>
  T *populate(const std::vector<T> &host) {
    T *d = alloc<T>(host.size());
    if (!host.empty()) check(pimdal_ingest(ctx, host.data(), sizeof(T) * host.size(), d, s), "pimdal_ingest");
    return d;
  }
  // get_results: the count from device memory, the error word, then the rows
  uint64_t count(const uint64_t *d_count) {
    uint64_t c = 0;
    check_cuda(cudaMemcpyAsync(&c, d_count, sizeof(c), cudaMemcpyDeviceToHost, s), "count");
    check(pimdal_ctx_sync_status(ctx, s), "pimdal_ctx_sync_status");
    return c;
  }
  template <class T>
  std::vector<T> fetch(const T *d, size_t n) {
    std::vector<T> h(n);
    if (n) check_cuda(cudaMemcpy(h.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost), "fetch");
    return h;
  }
};

void run_select(const std::string &dir, int64_t lo, int64_t hi) {
  Session x;
  const auto keys = read_file<int32_t>(dir + "/sel_keys.i32");
  const uint64_t n = keys.size();
  int32_t *d_keys = x.populate(keys);
  int32_t *d_vals = x.alloc<int32_t>(n);
  uint32_t *d_rows = x.alloc<uint32_t>(n);
  auto *d_res = x.alloc<pimdal_sel_results_t>(1);
  pimdal_sel_arguments_t a = {};
  a.size = n;
  a.in = d_keys;
  a.out = d_vals;
  a.out_ptr = d_rows;
  a.pred.op = PIMDAL_PRED_BETWEEN;
  a.pred.lo = lo;
  a.pred.hi = hi;
  a.key_dtype = PIMDAL_I32;
  a.layout = PIMDAL_LAYOUT_COLUMNS;
  check(pimdal_sel_kernel(x.ctx, &a, d_res, x.s), "pimdal_sel_kernel");
  const uint64_t c = x.count(&d_res->t_count);
  const auto vals = x.fetch(d_vals, c);
  const auto rows = x.fetch(d_rows, c);
  write_file(dir + "/sel_vals.i32", vals.data(), c);
  write_file(dir + "/sel_rows.u32", rows.data(), c);
}

void run_sort(const std::string &dir) {
  Session x;
  const auto keys = read_file<uint32_t>(dir + "/sort_keys.u32");
  const uint64_t n = keys.size();
  pimdal_sort_arguments_t a = {};
  a.nr_elements = n;
  a.in = x.populate(keys);
  a.out = x.alloc<uint32_t>(n);
  a.out_ptr = x.alloc<uint32_t>(n);
  a.key_dtype = PIMDAL_U32;
  a.layout = PIMDAL_LAYOUT_COLUMNS;
  size_t ws = 0;
  check(pimdal_sort_workspace_size(&a, &ws), "pimdal_sort_workspace_size");
  check(pimdal_ctx_set_workspace(x.ctx, x.alloc<char>(ws), ws), "pimdal_ctx_set_workspace");
  check(pimdal_sort_kernel(x.ctx, &a, x.s), "pimdal_sort_kernel");
  check(pimdal_ctx_sync_status(x.ctx, x.s), "pimdal_ctx_sync_status");
  const auto k = x.fetch(static_cast<uint32_t *>(a.out), n);
  const auto r = x.fetch(a.out_ptr, n);
  write_file(dir + "/sort_keys_out.u32", k.data(), n);
  write_file(dir + "/sort_rows.u32", r.data(), n);
}

void run_hash_join(const std::string &dir) {
  Session x;
  const auto bk = read_file<int32_t>(dir + "/hj_bk.i32");
  const auto bp = read_file<int32_t>(dir + "/hj_bp.i32");
  const auto pk = read_file<int32_t>(dir + "/hj_pk.i32");
  pimdal_hash_join_arguments_t a = {};
  a.build_key = x.populate(bk);
  a.build_payload = reinterpret_cast<const uint32_t *>(x.populate(bp));
  a.size_build = bk.size();
  a.probe_key = x.populate(pk);
  a.size_probe = pk.size();
  a.out_capacity = pk.size();
  a.out_build_payload = x.alloc<uint32_t>(pk.size());
  a.out_probe_ptr = x.alloc<uint32_t>(pk.size());
  size_t ws = 0;
  check(pimdal_hash_join_workspace_size(&a, &ws), "pimdal_hash_join_workspace_size");
  check(pimdal_ctx_set_workspace(x.ctx, x.alloc<char>(ws), ws), "pimdal_ctx_set_workspace");
  auto *d_res = x.alloc<pimdal_merge_results_t>(1);
  check(pimdal_hash_join(x.ctx, &a, d_res, x.s), "pimdal_hash_join");
  const uint64_t m = x.count(&d_res->t_count);
  const auto pay = x.fetch(a.out_build_payload, m);
  const auto row = x.fetch(a.out_probe_ptr, m);
  write_file(dir + "/hj_pay.u32", pay.data(), m);
  write_file(dir + "/hj_row.u32", row.data(), m);
}

void run_group_by(const std::string &dir) {
  Session x;
  const auto k = read_file<int32_t>(dir + "/gb_k.i32");
  const auto v = read_file<int64_t>(dir + "/gb_v.i64");
  const uint64_t n = k.size();
  pimdal_aggr_arguments_t a = {};
  a.size = n;
  a.in = x.populate(k);
  a.in_val = x.populate(v);
  a.out = x.alloc<int32_t>(n);
  a.out_sum = x.alloc<int64_t>(n);
  a.out_count = x.alloc<int64_t>(n);
  a.out_min = x.alloc<int64_t>(n);
  a.out_max = x.alloc<int64_t>(n);
  a.out_capacity = n;
  a.expected_groups = n;
  a.key_dtype = PIMDAL_I32;
  a.method = PIMDAL_GROUP_HASH;
  size_t ws = 0;
  check(pimdal_group_workspace_size(&a, &ws), "pimdal_group_workspace_size");
  check(pimdal_ctx_set_workspace(x.ctx, x.alloc<char>(ws), ws), "pimdal_ctx_set_workspace");
  auto *d_res = x.alloc<pimdal_aggr_results_t>(1);
  check(pimdal_group_kernel(x.ctx, &a, d_res, x.s), "pimdal_group_kernel");
  const uint64_t g = x.count(&d_res->t_count);
  write_file(dir + "/gb_key.i32", x.fetch(static_cast<int32_t *>(a.out), g).data(), g);
  write_file(dir + "/gb_sum.i64", x.fetch(a.out_sum, g).data(), g);
  write_file(dir + "/gb_count.i64", x.fetch(a.out_count, g).data(), g);
  write_file(dir + "/gb_min.i64", x.fetch(a.out_min, g).data(), g);
  write_file(dir + "/gb_max.i64", x.fetch(a.out_max, g).data(), g);
}

// TPC-H Q6 as the reference's pipeline runs it (pimdal/main/tpc_h/query6/
// dpu/kernel_q6.c:112-156: three selections, the product price * discount,
// the sum), here one pimdal_select_aggregate call over the resident columns.
void run_q6(const std::string &dir, int64_t date_lo, int64_t date_hi, int64_t quantity,
            int64_t discount) {
  Session x;
  const auto date = read_file<int32_t>(dir + "/q6_date.i32");
  const auto qty = read_file<int32_t>(dir + "/q6_qty.i32");
  const auto disc = read_file<int32_t>(dir + "/q6_disc.i32");
  const auto price = read_file<int64_t>(dir + "/q6_price.i64");
  pimdal_select_aggregate_arguments_t a = {};
  a.size = date.size();
  a.n_preds = 3;
  a.pred[0] = {x.populate(date), PIMDAL_I32, 0, {PIMDAL_PRED_RANGE, 0, date_lo, date_hi}};
  a.pred[1] = {x.populate(qty), PIMDAL_I32, 0, {PIMDAL_PRED_LT, 0, quantity, 0}};
  a.pred[2] = {x.populate(disc), PIMDAL_I32, 0,
               {PIMDAL_PRED_BETWEEN, 0, discount - 1, discount + 1}};
  a.key_space = 1;
  a.n_exprs = 1;
  a.expr[0].n_terms = 2;
  a.expr[0].term[0] = {x.populate(price), PIMDAL_I64, 0, 0};
  a.expr[0].term[1] = {a.pred[2].col, PIMDAL_I32, 0, 0};
  a.out_key = x.alloc<uint32_t>(1);
  a.out_count = x.alloc<int64_t>(1);
  a.out_sum[0] = x.alloc<int64_t>(1);
  a.out_capacity = 1;
  size_t ws = 0;
  check(pimdal_select_aggregate_workspace_size(&a, &ws), "pimdal_select_aggregate_workspace_size");
  check(pimdal_ctx_set_workspace(x.ctx, x.alloc<char>(ws), ws), "pimdal_ctx_set_workspace");
  auto *d_res = x.alloc<pimdal_aggr_results_t>(1);
  check(pimdal_select_aggregate(x.ctx, &a, d_res, x.s), "pimdal_select_aggregate");
  const uint64_t g = x.count(&d_res->t_count);
  int64_t out[2] = {0, 0};  // revenue, rows
  if (g) {
    out[0] = x.fetch(a.out_sum[0], 1)[0];
    out[1] = x.fetch(a.out_count, 1)[0];
  }
  write_file(dir + "/q6_out.i64", out, 2);
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 3) {
    std::fprintf(stderr,
                 "usage: %s <dir> select <lo> <hi> | sort | hash_join | group_by |"
                 " q6 <date_lo> <date_hi> <quantity> <discount>\n", argv[0]);
    return PIMDAL_ERR_ARG;
  }
  const std::string dir = argv[1], op = argv[2];
  try {
    if (op == "select" && argc == 5) run_select(dir, std::atoll(argv[3]), std::atoll(argv[4]));
    else if (op == "sort") run_sort(dir);
    else if (op == "hash_join") run_hash_join(dir);
    else if (op == "group_by") run_group_by(dir);
    else if (op == "q6" && argc == 7)
      run_q6(dir, std::atoll(argv[3]), std::atoll(argv[4]), std::atoll(argv[5]), std::atoll(argv[6]));
    else throw Failure{PIMDAL_ERR_ARG, "unknown operation " + op};
  } catch (const Failure &f) {
    std::fprintf(stderr, "%s: %s\n", f.where.c_str(), pimdal_status_string(f.status));
    return f.status;
  }
  return 0;
}
