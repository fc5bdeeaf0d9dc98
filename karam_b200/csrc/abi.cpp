// abi.cpp -- implementation of the C ABI (include/karam.h): contexts, problems,
// device buffers and the round driver that replays CUDA graphs of NR rounds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/karam.h"
#include "device.hpp"
#include "noalloc.hpp"
#include "seeder.hpp"
#include "topology.hpp"

using namespace karam;

namespace {

thread_local std::string g_create_error;

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw CudaError(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
}

// Owning device allocation.
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() {
    if (p) cudaFree(p);
  }
  void alloc(size_t b) {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = b;
    if (b) ck(cudaMalloc(&p, b), "cudaMalloc");
  }
  template <class T>
  T* as() const {
    return reinterpret_cast<T*>(p);
  }
};

template <class T>
void upload(DBuf& b, const std::vector<T>& v) {
  b.alloc(std::max<size_t>(v.size(), 1) * sizeof(T));
  if (!v.empty()) ck(cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
}

}  // namespace

struct karam_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  int max_smem = 0;
  std::string err;
};

struct karam_problem {
  karam_ctx* ctx = nullptr;
  Topology topo;
  int max_inst = 0;
  int ni = 0;
  bool inst_kp = false, inst_vth = false;  // per-instance MOSFET values present
  bool have_dc = false;
  int tuned[2] = {0, 0};  // measured factor/solve schedule per precision (0 = none)
  uint64_t content_hash = 0;  // karam_netlist_hash of the netlist the problem was made from
  int n_hub_items = 0, n_hub_slot_terms = 0;
  int max_hub_chunks = 0;  // k_es_one sums hub items of up to 8 chunks
  bool tran_started = false;  // capacitor history holds a transient in progress
  double t_now = 0.0, tran_h = 0.0;
  int tran_method = KARAM_TRAN_BE;

  // topology buffers
  DBuf t_mos_term, t_mos_geo, t_mos_pmos, t_dio_term, t_dio_par, t_res_term, t_res_g, t_cap_term,
      t_cap_c, t_mos_card, t_slot_rc, t_dio_lim, t_dio_level, t_vs_term, t_vs_kind, t_vs_pulse,
      t_is_term, t_is_amp, t_jlin, t_jcap_off, t_jcap_code, t_es_block, t_es_item, t_es_dev,
      t_es_jt, t_es_ft, t_es_fc, t_es_hub, t_es_hubc, t_lu_hdr, t_lu_data, t_lu_rec, t_lu_rec2, t_seed_vs, t_seed_anode,
      t_perm, t_slot_ptr, t_csc_ptr, t_csc_ent, t_mos_order, t_jt_off, t_jt_code, t_ft_off, t_ft_code,
      t_ft_a, t_ft_b, t_ft_coef, t_hub_items;
  DBuf t_nd[23];  // level schedule tables, in karam_get_lu_schedule's order
  DBuf t_nd_prog;  // the packed schedule (padded to whole int4)
  DevTopo dt{};
  // instance buffers, [item][ld] (instance-interleaved)
  int ld = 0;
  DBuf i_kp, i_vth, i_vsdc, i_v1, i_v2, i_v, i_x, i_F, i_J, i_cvp, i_cip, i_st, i_seed, i_out,
      i_redf, i_reddv, i_redfl, i_evt, i_evh,
      d_active, r_ws, r_list, r_count, i_vtp, i_vtpp, i_evl, d_counters, d_seed_ok, i_hub_part, i_hub_cnt, i_luws,
      i_live, i_stage, i_hist;
  cudaEvent_t ev_job0 = nullptr, ev_job1 = nullptr, ev_seed0 = nullptr, ev_seed1 = nullptr;
  bool seed_timed = false;  // ev_seed0 / ev_seed1 bracket this job's seeder inference
  int rescue_slots = 0;
  RescuePlan rplan;
  karam_seeder* seeder = nullptr;  // KARAM_SEED_MLP (not owned)
  DBuf i_feat;                     // [ni][n_features] FP32 seeder inputs
  int* h_active = nullptr;  // pinned

  // accounting of the last solve call
  karam_timing timing{};

  std::vector<int> csr_to_slot;  // CSR position -> value slot (-1: structurally zero)

  ~karam_problem() {
    if (h_active) cudaFreeHost(h_active);
    if (ev_job0) cudaEventDestroy(ev_job0);
    if (ev_job1) cudaEventDestroy(ev_job1);
    if (ev_seed0) cudaEventDestroy(ev_seed0);
    if (ev_seed1) cudaEventDestroy(ev_seed1);
  }
};

struct karam_seeder {
  karam_ctx* ctx = nullptr;
  karam::Mlp* m = nullptr;
  int n = 0, n_mos = 0, n_vs = 0, nv = 0;
  ~karam_seeder() {
    if (m) karam::mlp_destroy(m);
  }
};

namespace {

void set_err(karam_ctx* c, const std::string& m) {
  if (c)
    c->err = m;
  else
    g_create_error = m;
}

// Solves need a problem made with a context; a context-less problem carries
// only the host symbolic analysis.
void need_device(const karam_problem* p) {
  if (!p->ctx) throw std::logic_error("problem was created without a context (symbolic only)");
}

template <class F>
int guarded(karam_ctx* c, F f) {
  try {
    return f();
  } catch (const CudaError& e) {
    set_err(c, e.what());
    return KARAM_E_CUDA;
  } catch (const std::bad_alloc&) {
    set_err(c, "out of host memory");
    return KARAM_E_NOMEM;
  } catch (const std::logic_error& e) {
    set_err(c, e.what());
    return KARAM_E_STATE;
  } catch (const std::exception& e) {
    set_err(c, e.what());
    return KARAM_E_INVALID;
  }
}

void upload_topology(karam_problem* p) {
  const Topology& T = p->topo;
  std::vector<int4> mt;
  std::vector<double2> mg;
  std::vector<int> mp;
  std::vector<double2> mc;
  for (size_t i = 0; i < T.mos.size(); ++i) {
    mc.push_back(make_double2(T.mos[i].kp_card, T.mos[i].vto_card));
    mt.push_back(make_int4(T.mos_term[4 * i], T.mos_term[4 * i + 1], T.mos_term[4 * i + 2],
                           T.mos_term[4 * i + 3]));
    mg.push_back(make_double2(T.mos[i].wl, T.mos[i].lam));
    mp.push_back(T.mos[i].pmos ? 1 : 0);
  }
  std::vector<int2> dtm, rtm, ctm, vtm, itm;
  std::vector<double4> dpar;
  for (size_t i = 0; i < T.dio.size(); ++i) {
    dtm.push_back(make_int2(T.dio_term[2 * i], T.dio_term[2 * i + 1]));
    dpar.push_back(make_double4(T.dio[i].is, T.dio[i].n, T.dio[i].vt, 0.0));
  }
  std::vector<double> rg, cc, vpulse, ia;
  for (size_t i = 0; i < T.res.size(); ++i) {
    rtm.push_back(make_int2(T.res_term[2 * i], T.res_term[2 * i + 1]));
    rg.push_back(1.0 / T.res[i].val);
  }
  for (size_t i = 0; i < T.cap.size(); ++i) {
    ctm.push_back(make_int2(T.cap_term[2 * i], T.cap_term[2 * i + 1]));
    cc.push_back(T.cap[i].val);
  }
  std::vector<int> vk, seed_vs;
  for (size_t i = 0; i < T.vs.size(); ++i) {
    vtm.push_back(make_int2(T.vs_term[2 * i], T.vs_term[2 * i + 1]));
    vk.push_back(T.vs[i].kind);
    for (int k = 0; k < 7; ++k) vpulse.push_back(T.vs[i].pulse[k]);
    seed_vs.push_back(T.vs[i].pos > 0 ? T.iperm[T.vs[i].pos - 1] : -1);
  }
  for (size_t i = 0; i < T.isrc.size(); ++i) {
    itm.push_back(make_int2(T.is_term[2 * i], T.is_term[2 * i + 1]));
    ia.push_back(T.isrc[i].val);
  }
  std::vector<int> seed_an;
  for (int a : T.seed_anodes) seed_an.push_back(a > 0 ? T.iperm[a - 1] : -1);
  std::vector<int4> hdr;
  for (int k = 0; k < T.n; ++k)
    hdr.push_back(make_int4(T.lu_hdr[4 * k], T.lu_hdr[4 * k + 1], T.lu_hdr[4 * k + 2],
                            T.lu_hdr[4 * k + 3]));
  std::vector<double2> dlim;
  for (size_t i = 0; i < T.dio.size(); ++i)
    dlim.push_back(make_double2(T.dio_lim[2 * i], T.dio_lim[2 * i + 1]));

  upload(p->t_mos_term, mt);
  upload(p->t_mos_geo, mg);
  upload(p->t_mos_pmos, mp);
  upload(p->t_mos_card, mc);
  upload(p->t_dio_term, dtm);
  upload(p->t_dio_par, dpar);
  upload(p->t_dio_lim, dlim);
  upload(p->t_dio_level, T.dio_level);
  upload(p->t_res_term, rtm);
  upload(p->t_res_g, rg);
  upload(p->t_cap_term, ctm);
  upload(p->t_cap_c, cc);
  upload(p->t_vs_term, vtm);
  upload(p->t_vs_kind, vk);
  upload(p->t_vs_pulse, vpulse);
  upload(p->t_is_term, itm);
  upload(p->t_is_amp, ia);
  upload(p->t_jlin, T.jlin_dc);
  upload(p->t_jcap_off, T.jcap_off);
  upload(p->t_jcap_code, T.jcap_code);
  {
    auto int4s = [](const std::vector<int>& v) {
      std::vector<int4> o(v.size() / 4);
      for (size_t k = 0; k < o.size(); ++k) o[k] = make_int4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
      return o;
    };
    upload(p->t_es_block, int4s(T.es_block));
    upload(p->t_es_hubc, int4s(T.es_hubc));
    upload(p->t_es_item, int4s(T.es_item));
    upload(p->t_es_ft, int4s(T.es_ft));
  }
  upload(p->t_es_dev, T.es_dev);
  upload(p->t_es_jt, T.es_jt);
  upload(p->t_es_fc, T.es_fc);
  upload(p->t_es_hub, T.es_hub);
  upload(p->t_lu_hdr, hdr);
  upload(p->t_lu_data, T.lu_data);
  upload(p->t_lu_rec, T.lu_rec);
  upload(p->t_lu_rec2, T.lu_rec2);
  upload(p->t_seed_vs, seed_vs);
  upload(p->t_seed_anode, seed_an);
  upload(p->t_perm, T.perm);
  upload(p->t_mos_order, T.mos_order);
  upload(p->t_jt_off, T.jt_off);
  upload(p->t_jt_code, T.jt_code);
  upload(p->t_ft_off, T.ft_off);
  upload(p->t_ft_code, T.ft_code);
  upload(p->t_ft_a, T.ft_a);
  upload(p->t_ft_b, T.ft_b);
  upload(p->t_ft_coef, T.ft_coef);
  {
    // hub items from the chunk-0 block of each hub group
    std::vector<int4> hubs;
    p->n_hub_slot_terms = 0;
    for (size_t b = 0; b < T.es_block.size() / 4; ++b)
      if (T.es_block[4 * b + 1] < 0 && T.es_hubc[4 * b] == 0)
        for (int m = 0; m < -T.es_block[4 * b + 1]; ++m) {
          const int k = T.es_block[4 * b] + m, it = T.es_item[4 * k];
          hubs.push_back(make_int4(it, T.es_item[4 * k + 3], T.es_hubc[4 * b + 1], p->n_hub_slot_terms));
          if (it < T.nv) p->n_hub_slot_terms += T.jt_off[it + 1] - T.jt_off[it];
        }
    upload(p->t_hub_items, hubs);
    p->n_hub_items = (int)hubs.size();
    p->max_hub_chunks = 0;
    for (const int4& h : hubs) p->max_hub_chunks = std::max(p->max_hub_chunks, h.z);
  }
  std::vector<int2> src;
  for (int s = 0; s < T.nv; ++s) src.push_back(make_int2(T.slot_row[s], T.slot_col[s]));
  upload(p->t_slot_rc, src);
  // value slots by row (row-major numbering, columns ascending) and by column
  std::vector<int> slot_ptr(T.n + 1, 0), csc_ptr(T.n + 1, 0);
  for (int s = 0; s < T.nv; ++s) {
    slot_ptr[T.slot_row[s] + 1]++;
    csc_ptr[T.slot_col[s] + 1]++;
  }
  for (int i = 0; i < T.n; ++i) {
    slot_ptr[i + 1] += slot_ptr[i];
    csc_ptr[i + 1] += csc_ptr[i];
  }
  std::vector<int2> csc_ent(T.nv);
  {
    std::vector<int> fillp(csc_ptr.begin(), csc_ptr.end() - 1);
    for (int s = 0; s < T.nv; ++s) csc_ent[fillp[T.slot_col[s]]++] = make_int2(T.slot_row[s], s);
  }
  upload(p->t_slot_ptr, slot_ptr);
  upload(p->t_csc_ptr, csc_ptr);
  upload(p->t_csc_ent, csc_ent);

  DevTopo& d = p->dt;
  d.n = T.n;
  d.nv = T.nv;
  d.n_mos = (int)T.mos.size();
  d.n_dio = (int)T.dio.size();
  d.n_res = (int)T.res.size();
  d.n_cap = (int)T.cap.size();
  d.n_vs = (int)T.vs.size();
  d.n_is = (int)T.isrc.size();
  d.temp_k = T.temp_k;
  d.mos_term = p->t_mos_term.as<int4>();
  d.mos_geo = p->t_mos_geo.as<double2>();
  d.mos_pmos = p->t_mos_pmos.as<int>();
  d.mos_card = p->t_mos_card.as<double2>();
  d.dio_term = p->t_dio_term.as<int2>();
  d.dio_par = p->t_dio_par.as<double4>();
  d.dio_lim = p->t_dio_lim.as<double2>();
  d.dio_level = p->t_dio_level.as<int>();
  d.n_dio_levels = T.n_dio_levels;
  d.res_term = p->t_res_term.as<int2>();
  d.res_g = p->t_res_g.as<double>();
  d.cap_term = p->t_cap_term.as<int2>();
  d.cap_c = p->t_cap_c.as<double>();
  d.vs_term = p->t_vs_term.as<int2>();
  d.vs_kind = p->t_vs_kind.as<int>();
  d.vs_pulse = p->t_vs_pulse.as<double>();
  d.is_term = p->t_is_term.as<int2>();
  d.is_amp = p->t_is_amp.as<double>();
  d.jlin_dc = p->t_jlin.as<double>();
  d.jcap_off = p->t_jcap_off.as<int>();
  d.jcap_code = p->t_jcap_code.as<int>();
  d.n_es_blocks = (int)T.es_block.size() / 4;
  d.es_block = p->t_es_block.as<int4>();
  d.es_item = p->t_es_item.as<int4>();
  d.es_dev = p->t_es_dev.as<int>();
  d.es_jt = p->t_es_jt.as<int>();
  d.es_ft = p->t_es_ft.as<int4>();
  d.es_fc = p->t_es_fc.as<double>();
  d.es_hub = p->t_es_hub.as<int>();
  d.es_hubc = p->t_es_hubc.as<int4>();
  d.jt_off = p->t_jt_off.as<int>();
  d.jt_code = p->t_jt_code.as<int>();
  d.ft_off = p->t_ft_off.as<int>();
  d.ft_code = p->t_ft_code.as<int>();
  d.ft_a = p->t_ft_a.as<int>();
  d.ft_b = p->t_ft_b.as<int>();
  d.ft_coef = p->t_ft_coef.as<double>();
  d.hub_items = p->t_hub_items.as<int4>();
  d.n_hub_items = p->n_hub_items;
  d.n_ft_terms = T.ft_off.empty() ? 0 : T.ft_off.back();
  d.n_hub_slot_terms = p->n_hub_slot_terms;
  d.n_jt_terms = T.jt_off.empty() ? 0 : T.jt_off.back();
  d.n_hub_groups = T.n_hub_groups;
  d.n_hub_rows = T.n_hub_rows;
  d.lu_hdr = p->t_lu_hdr.as<int4>();
  d.lu_data = p->t_lu_data.as<int>();
  d.lu_small = T.lu_small ? 1 : 0;
  d.lu_rec = T.lu_small ? p->t_lu_rec.as<int4>() : nullptr;
  d.lu_rec2 = T.lu_small ? p->t_lu_rec2.as<int2>() : nullptr;
  d.slot_rc = p->t_slot_rc.as<int2>();
  d.nd_levels = T.nd_levels;
  d.nd_nv = T.nd_nv;
  d.nd_S = T.nd_nv | 1;
  d.nd_SY = T.n | 1;
  if (T.nd_levels > 0) {
    const std::vector<int>* tabs[23] = {
        &T.nd_pos, &T.nd_src, &T.nd_diag, &T.lv_piv, &T.lv_piv_ptr, &T.lv_l_ptr, &T.l_slot,
        &T.l_piv, &T.lv_ts_ptr, &T.lv_tl_ptr, &T.t_slot, &T.t_off, &T.pr_l, &T.pr_u, &T.lv_ys_ptr,
        &T.lv_yl_ptr, &T.y_row, &T.y_off, &T.yp_l, &T.yp_k, &T.bs_off, &T.bs_u, &T.bs_c};
    const int** dst[23] = {&d.nd_pos, &d.nd_src, &d.nd_diag, &d.lv_piv, &d.lv_piv_ptr,
                           &d.lv_l_ptr, &d.l_slot, &d.l_piv, &d.lv_ts_ptr, &d.lv_tl_ptr,
                           &d.t_slot, &d.t_off, &d.pr_l, &d.pr_u, &d.lv_ys_ptr, &d.lv_yl_ptr,
                           &d.y_row, &d.y_off, &d.yp_l, &d.yp_k, &d.bs_off, &d.bs_u, &d.bs_c};
    for (int t = 0; t < 23; ++t) {
      std::vector<int> v = *tabs[t];
      if (v.empty()) v.push_back(0);
      upload(p->t_nd[t], v);
      *dst[t] = p->t_nd[t].as<int>();
    }
  }
  d.nd_prog = nullptr;
  d.nd_prog_len = 0;
  if (!T.nd_prog.empty()) {
    std::vector<int> pg = T.nd_prog;
    pg.resize((pg.size() + 3) / 4 * 4, 0);
    upload(p->t_nd_prog, pg);
    d.nd_prog = p->t_nd_prog.as<int>();
    d.nd_prog_len = (int)pg.size();
  }
  d.slot_ptr = p->t_slot_ptr.as<int>();
  d.csc_ptr = p->t_csc_ptr.as<int>();
  d.csc_ent = p->t_csc_ent.as<int2>();
  d.seed_vs = p->t_seed_vs.as<int>();
  d.seed_anode = p->t_seed_anode.as<int>();
  d.n_seed_anode = (int)seed_an.size();

  // CSR position -> value slot (for karam_eval_stamp)
  p->csr_to_slot.assign(T.nnz(), -1);
  for (size_t k = 0; k < T.trip.size(); ++k) p->csr_to_slot[T.slot_csr[k]] = T.f_slot[T.trip[k].f];
}

void alloc_instances(karam_problem* p) {
  const Topology& T = p->topo;
  const size_t M = (size_t)p->max_inst, n = T.n, nm = T.mos.size(), nv = T.vs.size();
  p->ld = lane_stride(p->max_inst);
  const size_t ld = (size_t)p->ld;
  p->i_kp.alloc(std::max<size_t>(1, ld * nm) * sizeof(float));
  p->i_vth.alloc(std::max<size_t>(1, ld * nm) * sizeof(float));
  p->i_vsdc.alloc(std::max<size_t>(1, ld * nv) * sizeof(double));
  p->i_v1.alloc(std::max<size_t>(1, ld * nv) * sizeof(double));
  p->i_v2.alloc(std::max<size_t>(1, ld * nv) * sizeof(double));
  p->i_v.alloc(ld * n * sizeof(double));
  p->i_x.alloc(ld * n * sizeof(double));
  p->i_F.alloc(ld * n * sizeof(double));
  p->i_J.alloc(std::max<size_t>(1, ld * (size_t)T.nv) * sizeof(double));
  p->i_redf.alloc(ld * sizeof(unsigned long long));
  p->i_reddv.alloc(ld * sizeof(unsigned long long));
  p->i_redfl.alloc(ld * sizeof(int));
  p->i_evt.alloc(ld * sizeof(double));
  p->i_evh.alloc(ld * sizeof(double));
  p->i_hub_part.alloc(std::max<size_t>(1, ld * (size_t)T.n_hub_rows) * sizeof(double));
  p->i_hub_cnt.alloc(std::max<size_t>(1, ld / 32 * (size_t)T.n_hub_groups) * sizeof(int));
  ck(cudaMemset(p->i_hub_cnt.p, 0, std::max<size_t>(1, ld / 32 * (size_t)T.n_hub_groups) * sizeof(int)),
     "memset hub counters");
  {
    // lanes beyond the batch never evaluate
    std::vector<double> neg(ld, -1.0);
    ck(cudaMemcpy(p->i_evh.p, neg.data(), ld * sizeof(double), cudaMemcpyHostToDevice), "init ev");
  }
  p->i_cvp.alloc(std::max<size_t>(1, ld * T.cap.size()) * sizeof(double));
  p->i_cip.alloc(std::max<size_t>(1, ld * T.cap.size()) * sizeof(double));
  p->i_st.alloc(M * sizeof(InstState));
  p->i_hist.alloc(ld * 2 * KHIST_LEN * sizeof(double));
  p->i_seed.alloc(ld * n * sizeof(double));
  p->i_vtp.alloc(ld * n * sizeof(double));
  p->i_vtpp.alloc(ld * n * sizeof(double));
  upload(p->i_evl, std::vector<double>(ld, -1.0));
  p->i_out.alloc(ld * n * sizeof(double));
  p->d_active.alloc(2 * sizeof(int));  // live instances; most rounds of a persistent launch
  p->d_seed_ok.alloc(sizeof(int));
  p->d_counters.alloc(5 * sizeof(unsigned long long));
  ck(cudaEventCreate(&p->ev_job0), "cudaEventCreate");
  ck(cudaEventCreate(&p->ev_job1), "cudaEventCreate");
  ck(cudaEventCreate(&p->ev_seed0), "cudaEventCreate");
  ck(cudaEventCreate(&p->ev_seed1), "cudaEventCreate");
  // Partial-pivoting rescue: per concurrently running rescue warp, the U
  // factor and room for rows with fill (2 n x n FP64), within a 2 GiB budget.
  p->rplan = plan_rescue(p->dt);
  p->rplan.ctas_per_sm = rescue_ctas_per_sm(p->dt, p->rplan);
  const size_t per = 2 * n * n * sizeof(double);
  const size_t budget = size_t(2) << 30;
  const size_t resident =
      (size_t)p->rplan.warps * p->rplan.ctas_per_sm * std::max(1, p->ctx->num_sms);
  // no rescue when its slot tables do not fit a CTA's shared memory (large
  // problems): a failed solve then aborts the step as in the reference
  size_t slots = p->rplan.warps > 0 ? std::min<size_t>({M, resident, budget / per}) : 0;
  // whole CTAs: every warp of the grid takes items (item e on CTA e % grid)
  if (slots >= (size_t)p->rplan.warps && p->rplan.warps > 0)
    slots -= slots % p->rplan.warps;
  else if (slots > 0)
    p->rplan.warps = (int)slots;
  p->rescue_slots = (int)slots;
  if (slots > 0) {
    p->r_ws.alloc(slots * per);
    p->r_list.alloc(M * sizeof(RescueItem));
    p->r_count.alloc(sizeof(int));
    ck(cudaMemset(p->r_count.p, 0, sizeof(int)), "memset rescue count");
  }
  ck(cudaMallocHost(&p->h_active, 2 * sizeof(int)), "cudaMallocHost");
}

DevInst dev_inst(karam_problem* p) {
  DevInst I{};
  I.ni = p->ni;
  I.ld = p->ld;
  I.kp = p->inst_kp ? p->i_kp.as<float>() : nullptr;
  I.vth = p->inst_vth ? p->i_vth.as<float>() : nullptr;
  I.vs_dc = p->i_vsdc.as<double>();
  I.vs_v1 = p->i_v1.as<double>();
  I.vs_v2 = p->i_v2.as<double>();
  I.v = p->i_v.as<double>();
  I.x = p->i_x.as<double>();
  I.F = p->i_F.as<double>();
  I.J = p->i_J.p;
  I.red_f = p->i_redf.as<unsigned long long>();
  I.red_dv = p->i_reddv.as<unsigned long long>();
  I.red_flags = p->i_redfl.as<int>();
  I.ev_t = p->i_evt.as<double>();
  I.ev_heff = p->i_evh.as<double>();
  I.cap_vp = p->i_cvp.as<double>();
  I.cap_ip = p->i_cip.as<double>();
  I.v_tp = p->i_vtp.as<double>();
  I.v_tpp = p->i_vtpp.as<double>();
  I.ev_lte = p->i_evl.as<double>();
  I.st = p->i_st.as<InstState>();
  I.hist = p->i_hist.as<double>();
  I.seed = nullptr;
  I.rescue_ws = p->rescue_slots > 0 ? p->r_ws.as<double>() : nullptr;
  I.rescue_list = p->rescue_slots > 0 ? p->r_list.as<RescueItem>() : nullptr;
  I.rescue_count = p->rescue_slots > 0 ? p->r_count.as<int>() : nullptr;
  I.rescue_slots = p->rescue_slots;
  I.hub_part = p->i_hub_part.as<double>();
  I.hub_cnt = p->i_hub_cnt.as<int>();
  I.counters = p->d_counters.as<unsigned long long>();
  I.wave = nullptr;
  I.wave_pos = nullptr;
  I.n_wave = 0;
  I.wave_steps = 0;
  return I;
}

void set_instances_impl(karam_problem* p, const karam_instances* inst) {
  const Topology& T = p->topo;
  int ni = inst ? inst->n_instances : 1;
  if (ni < 1 || ni > p->max_inst) throw std::runtime_error("n_instances out of range");
  const size_t nm = T.mos.size(), nv = T.vs.size(), ld = (size_t)p->ld;
  // instance-interleaved: item k of instance i at [k * ld + i]. Per-instance
  // KP / VTO go to the device as the caller laid them out ([instance][MOSFET],
  // netlist order) and are interleaved there; model-card values and the
  // sources are laid out here.
  const bool dev_kp = inst && inst->mos_kp, dev_vth = inst && inst->mos_vto;
  std::vector<float> kp(dev_kp ? 0 : ld * nm, 0.0f), vth(dev_vth ? 0 : ld * nm, 0.0f);
  std::vector<double> vdc(ld * nv, 0.0), v1(ld * nv, 0.0), v2(ld * nv, 0.0);
  for (int i = 0; i < ni; ++i) {
    for (size_t j = 0; j < nm && !(dev_kp && dev_vth); ++j) {
      if (!dev_kp) kp[j * ld + i] = (float)T.mos[j].kp_card;
      if (!dev_vth) vth[j * ld + i] = (float)T.mos[j].vto_card;
    }
    for (size_t s = 0; s < nv; ++s) {
      const auto& V = T.vs[s];
      double dc = V.dc, sc = 1.0;
      if (inst && inst->vs_dc) {
        dc = inst->vs_dc[(size_t)i * nv + s];
        if (V.dc != 0.0) sc = dc / V.dc;
      }
      vdc[s * ld + i] = dc;
      v1[s * ld + i] = V.kind == KARAM_SRC_PULSE ? V.pulse[0] * sc : dc;
      v2[s * ld + i] = V.kind == KARAM_SRC_PULSE ? V.pulse[1] * sc : dc;
    }
  }
  // Without per-instance values the kernel reads the FP64 model-card table.
  p->inst_kp = inst && inst->mos_kp;
  p->inst_vth = inst && inst->mos_vto;
  cudaStream_t s = p->ctx->stream;
  if (nm) {
    const size_t rows = (size_t)ni * nm;
    if ((dev_kp || dev_vth) && p->i_stage.bytes < 2 * (size_t)p->max_inst * nm * sizeof(float))
      p->i_stage.alloc(2 * (size_t)p->max_inst * nm * sizeof(float));
    float* stage = p->i_stage.as<float>();
    auto put = [&](bool dev, const float* src, const std::vector<float>& host, DBuf& dst, float* stg,
                   const char* what) {
      if (dev) {
        ck(cudaMemcpyAsync(stg, src, rows * sizeof(float), cudaMemcpyHostToDevice, s), what);
        interleave_f(stg, p->t_mos_order.as<int>(), dst.as<float>(), ni, (int)ld, (int)nm, s);
        ck(cudaGetLastError(), "k_interleave_f launch");
      } else {
        ck(cudaMemcpyAsync(dst.p, host.data(), host.size() * sizeof(float), cudaMemcpyHostToDevice, s),
           what);
      }
    };
    put(dev_kp, dev_kp ? inst->mos_kp : nullptr, kp, p->i_kp, stage, "H2D kp");
    put(dev_vth, dev_vth ? inst->mos_vto : nullptr, vth, p->i_vth,
        stage + (size_t)p->max_inst * nm, "H2D vth");
  }
  if (nv) {
    ck(cudaMemcpyAsync(p->i_vsdc.p, vdc.data(), vdc.size() * sizeof(double), cudaMemcpyHostToDevice, s), "H2D vs");
    ck(cudaMemcpyAsync(p->i_v1.p, v1.data(), v1.size() * sizeof(double), cudaMemcpyHostToDevice, s), "H2D v1");
    ck(cudaMemcpyAsync(p->i_v2.p, v2.data(), v2.size() * sizeof(double), cudaMemcpyHostToDevice, s), "H2D v2");
  }
  ck(cudaStreamSynchronize(s), "set_instances sync");
  p->ni = ni;
  p->have_dc = false;
}

JobParams job_params(const karam_solver_opts* o, int n_steps, double h, int method) {
  JobParams P{};
  karam_solver_opts d;
  karam_default_opts(&d);
  if (!o) o = &d;
  P.precision = o->precision;
  P.max_nr_iter = o->max_nr_iter;
  P.gmin_steps = o->gmin_steps;
  P.reltol = o->reltol;
  P.vntol = o->vntol;
  P.kcl_shortcut = o->kcl_shortcut;
  P.kcl_tol = o->kcl_tol;
  P.polish_max = o->polish_max;
  P.polish_rel = o->polish_rel;
  P.polish_abs = o->polish_abs;
  P.lte_rel = o->lte_reltol > 0.0 ? o->lte_reltol : 0.0;
  P.lte_abs = o->lte_abstol;
  P.n_steps = n_steps;
  P.h = h;
  P.method = method;
  P.seeded = o->seeded;
  P.seed_max_iter = o->seed_max_iter;
  P.seed_bcast = 0;
  if (P.seeded < KARAM_SEED_NONE || P.seeded > KARAM_SEED_MLP)
    throw std::runtime_error("unknown seeded mode");
  P.max_halvings = o->max_halvings;
  P.growth32 = o->lu_growth_limit > 0 ? o->lu_growth_limit : (o->lu_growth_limit < 0 ? 1e300 : 1e4);
  P.growth64 = o->lu_growth_limit > 0 ? o->lu_growth_limit : (o->lu_growth_limit < 0 ? 1e300 : 1e10);
  if (P.max_halvings < 0 || P.max_halvings > 10) throw std::runtime_error("max_halvings must be in 0..10");
  if (P.max_nr_iter < 1 || P.gmin_steps < 1 || P.polish_max < 0)
    throw std::runtime_error("invalid solver options");
  if (P.precision != KARAM_PREC_FP64 && P.precision != KARAM_PREC_MIXED)
    throw std::runtime_error("unknown precision");
  if (n_steps > 0 && !(h > 0)) throw std::runtime_error("transient step must be > 0");
  if (method != KARAM_TRAN_BE && method != KARAM_TRAN_TRAP) throw std::runtime_error("unknown method");
  return P;
}

// Measured schedules (karam_tune_schedule), per problem and process-wide by
// netlist content (karam_netlist_hash), device, batch size and precision: a
// schedule is reused only for the same topology on the same GPU, since the
// shared memory a schedule needs depends on the topology and what fits
// depends on the device.
using TuneKey = std::tuple<uint64_t, int, int, int>;
std::mutex g_tune_mu;
std::map<TuneKey, int>& tune_cache() {
  static std::map<TuneKey, int> m;
  return m;
}
TuneKey tune_key(const karam_problem* p, int prec) {
  return TuneKey{p->content_hash, p->ctx ? p->ctx->device : -1, p->ni, prec};
}
// The schedule option a solve with opts.schedule == 0 uses: the problem's
// measured choice, else one measured for an identical netlist and batch size
// on the same device, else 0 (the planner's).
int tuned_schedule(const karam_problem* p, int prec) {
  const int idx = prec == KARAM_PREC_MIXED ? 1 : 0;
  if (p->tuned[idx]) return p->tuned[idx];
  std::lock_guard<std::mutex> lock(g_tune_mu);
  const auto it = tune_cache().find(tune_key(p, prec));
  return it == tune_cache().end() ? 0 : it->second;
}

// Runs NR rounds until every instance is done (or opts->max_rounds ends).
// Rounds (k_es, k_lu, k_rescue) are captured in a CUDA graph of kRounds
// rounds; the last k_lu of the graph counts the live instances into d_active,
// which is read back after every replay. k_es resets the rescue counter of its
// round, so the graph holds kernels only (and one memset per replay). With
// opts->kernel_timing, event records between the kernels time each of them;
// they are left out otherwise, since they cost more than the empty launches
// of a round.
//
// Tail: once no more instances are live than the GPU has SMs, a problem on
// the warp-per-instance level schedule switches to a second graph in which
// k_lu_big gives each live instance a CTA of its own, over a list of the live
// instances that the kernel itself refreshes every round (two lists, in turn).
// k_lu_big runs the same arithmetic as k_lu_nd, so the results do not change;
// a round with one live instance takes well under half the time.
void run_rounds(karam_problem* p, const JobParams& P, const karam_solver_opts* opts,
                const DevInst* inst = nullptr) {
  constexpr int kRounds = 16;  // even: the tail rounds alternate between two lists
  const int max_rounds = opts ? opts->max_rounds : 0;
  int want_lanes = opts ? opts->schedule : 0;
  const bool from_tuner = want_lanes == 0;
  if (from_tuner) want_lanes = tuned_schedule(p, P.precision);
  const bool timed = opts && opts->kernel_timing;
  cudaStream_t s = p->ctx->stream;
  DevInst I = inst ? *inst : dev_inst(p);
  const int prec = P.precision;
  const int max_smem = p->ctx->max_smem, num_sms = p->ctx->num_sms;
  // the per-round graph's plan (the planner's choice under the persistent option)
  RoundLaunch L = plan_round(p->dt, p->ni, prec, max_smem, num_sms, want_lanes == -4 ? 0 : want_lanes);
  if (L.L < 1 && from_tuner && want_lanes != 0) {
    // a measured schedule that does not fit here falls back to the planner's choice
    cudaGetLastError();
    L = plan_round(p->dt, p->ni, prec, max_smem, num_sms, 0);
  }
  if (L.L < 1)
    throw std::runtime_error(std::string("no factor/solve schedule fits this problem; last: ") + L.why);
  ck(cudaGetLastError(), "configure kernels");
  p->timing.lanes = L.L;
  p->timing.level_schedule = L.big == 5 ? 6 : L.big ? 1 + L.big : L.nd ? 1 : 0;
  RoundLaunch LT;  // the tail's block-per-instance plan (L == 0: no tail switch)
  if (L.nd && p->ni > num_sms) {  // L.nd: the packed program exists
    LT = plan_round(p->dt, p->ni, prec, max_smem, num_sms, -3);
    cudaGetLastError();
  }
  // The persistent per-instance kernel runs an instance's remaining rounds in
  // one launch with the code of the per-instance round kernels: for batches
  // no larger than the SM count (opts.schedule 0 or -4) and for the tail once
  // no more instances are live than SMs. Each CTA rescues its own failed
  // solves, so the rescue workspace must have a slot per CTA.
  const int want = want_lanes;  // after the measured choice
  PersistPlan pplan;
  if (!timed && p->max_hub_chunks <= 8) {
    pplan = plan_persist(p->dt, prec, p->rplan, max_smem);
    cudaGetLastError();
  }
  auto persist_fits = [&](int grid) {
    return pplan.smem > 0 && (p->rescue_slots == 0 || p->rescue_slots >= grid);
  };
  const int budget = max_rounds > 0 ? max_rounds : (1 << 30);
  int* active = p->d_active.as<int>();
  // all rounds of every instance in one launch
  auto run_persist = [&](const DevInst& Ip, int grid, int rounds_left, bool is_tail) {
    ck(cudaMemsetAsync(active, 0, 2 * sizeof(int), s), "memset active");
    launch_persist(p->dt, Ip, P, prec, grid, pplan, rounds_left, p->rplan.K, active, active + 1, s);
    ck(cudaGetLastError(), "k_persist launch");
    ck(cudaMemcpyAsync(p->h_active, active, 2 * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H active");
    ck(cudaStreamSynchronize(s), "persistent sync");
    ++p->timing.other_launches;
    p->timing.rounds += p->h_active[1];
    p->timing.persistent_rounds += p->h_active[1];
    if (pplan.resident_at > 0) p->timing.resident_instances += grid;
    if (is_tail) p->timing.tail_rounds += p->h_active[1];
  };
  if (want == -4 && !persist_fits(p->ni))
    throw std::runtime_error("the persistent per-instance schedule does not fit this problem");
  if (want == -4 || (want == 0 && p->ni <= num_sms && persist_fits(p->ni))) {
    p->timing.lanes = 1;
    p->timing.level_schedule = 5;
    run_persist(I, p->ni, budget, false);
    return;
  }
  if (L.big == 2 || L.big == 5) {  // the ND slots of every instance in global memory
    const size_t per = (size_t)p->dt.nd_S + (L.big == 5 ? (size_t)p->dt.nd_SY : 0);  // 5: + the solve vector
    const size_t need = (size_t)p->ni * per * sizeof(double);
    if (p->i_luws.bytes < need) p->i_luws.alloc(need);
    I.lu_ws = p->i_luws.p;
  }
  std::vector<cudaEvent_t> ev(timed ? 4 * kRounds : 0);
  for (auto& e : ev) ck(cudaEventCreate(&e), "cudaEventCreate");
  struct EvGuard {
    std::vector<cudaEvent_t>& v;
    ~EvGuard() {
      for (auto e : v) cudaEventDestroy(e);
    }
  } eg{ev};

  struct Graph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ~Graph() {
      if (e) cudaGraphExecDestroy(e);
      if (g) cudaGraphDestroy(g);
    }
  };
  // kRounds rounds on plan Lp, round r with the instances of Iv[r % 2]
  auto capture = [&](Graph& G, const RoundLaunch& Lp, const DevInst* Iv) {
    ck(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture");
    // External event records become event-record nodes of the graph (a plain
    // record inside capture would only order work within the capture); a
    // launch that fails inside the capture is reported by name
    const char* failed = nullptr;
    cudaError_t launch_err = cudaSuccess;
    auto check = [&](const char* what) {
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess && launch_err == cudaSuccess) {
        launch_err = e;
        failed = what;
      }
    };
    for (int r = 0; r < kRounds; ++r) {
      const DevInst& Ir = Iv[r & 1];
      if (r == kRounds - 1) cudaMemsetAsync(active, 0, sizeof(int), s);
      if (timed) cudaEventRecordWithFlags(ev[4 * r], s, cudaEventRecordExternal);
      launch_eval_stamp(p->dt, Ir, P, Lp, prec, s);
      check("k_es launch");
      if (timed) cudaEventRecordWithFlags(ev[4 * r + 1], s, cudaEventRecordExternal);
      launch_lu(p->dt, Ir, P, Lp, prec, active, s);
      check("k_lu launch");
      if (timed) cudaEventRecordWithFlags(ev[4 * r + 2], s, cudaEventRecordExternal);
      if (Ir.rescue_list) launch_rescue(p->dt, Ir, P, p->rplan, s);
      check("k_rescue launch");
      if (timed) cudaEventRecordWithFlags(ev[4 * r + 3], s, cudaEventRecordExternal);
    }
    const cudaError_t end_err = cudaStreamEndCapture(s, &G.g);
    ck(launch_err, failed ? failed : "kernel launch in capture");
    ck(end_err, "end capture");
    ck(cudaGraphInstantiate(&G.e, G.g, 0), "graph instantiate");
  };
  Graph main_g, tail_g;
  const DevInst Im[2] = {I, I};
  capture(main_g, L, Im);
  bool tail = false;

  while (true) {
    ck(cudaGraphLaunch(tail ? tail_g.e : main_g.e, s), "graph launch");
    ck(cudaMemcpyAsync(p->h_active, active, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H active");
    ck(cudaStreamSynchronize(s), "round sync");
    for (int r = 0; r < kRounds && timed; ++r) {
      float a = 0, b = 0, c = 0;
      ck(cudaEventElapsedTime(&a, ev[4 * r], ev[4 * r + 1]), "event time");
      ck(cudaEventElapsedTime(&b, ev[4 * r + 1], ev[4 * r + 2]), "event time");
      ck(cudaEventElapsedTime(&c, ev[4 * r + 2], ev[4 * r + 3]), "event time");
      p->timing.eval_ms += a;
      p->timing.lu_ms += b;
      p->timing.rescue_ms += c;
    }
    p->timing.eval_launches += kRounds;
    p->timing.lu_launches += kRounds;
    if (I.rescue_list) p->timing.rescue_launches += kRounds;
    p->timing.rounds += kRounds;
    if (tail) p->timing.tail_rounds += kRounds;
    if (*p->h_active == 0 || p->timing.rounds >= budget) break;
    if (!tail && LT.L > 0 && *p->h_active <= num_sms) {
      // lists: [count 0, count 1, pad to 16 B, list 0 [ni], list 1 [ni]]
      const size_t need = sizeof(int) * (4 + 2 * (size_t)p->ni);
      if (p->i_live.bytes < need) p->i_live.alloc(need);
      int* cnt = p->i_live.as<int>();
      int* list0 = cnt + 4;
      int* list1 = list0 + p->ni;
      ck(cudaMemsetAsync(cnt, 0, 2 * sizeof(int), s), "memset live counts");
      launch_live_list(I, list0, cnt, s);
      ck(cudaGetLastError(), "k_live_list launch");
      ++p->timing.other_launches;
      DevInst It[2] = {I, I};
      It[0].live_in = list0;
      It[0].live_in_count = cnt;
      It[0].live_out = list1;
      It[0].live_out_count = cnt + 1;
      It[1].live_in = list1;
      It[1].live_in_count = cnt + 1;
      It[1].live_out = list0;
      It[1].live_out_count = cnt;
      LT.grid = *p->h_active;  // instances only ever leave the live set
      if (persist_fits(LT.grid)) {  // the remaining rounds of every live instance in one launch
        DevInst Ip = I;
        Ip.live_in = list0;
        Ip.live_in_count = cnt;
        run_persist(Ip, LT.grid, budget - p->timing.rounds, true);
        break;
      }
      // the per-instance evaluation kernel, when its device values fit the
      // default 48 KiB of dynamic shared memory and its hubs 8 chunks
      LT.es_one = p->max_hub_chunks <= 8 &&
                  sizeof(double) * (3 * (size_t)(p->dt.n_mos + p->dt.n_dio) + (size_t)p->dt.n_ft_terms +
                                    (size_t)p->dt.n_hub_slot_terms) <= 48 * 1024;
      capture(tail_g, LT, It);
      tail = true;
    }
  }
}

// The recorded DC convergence history of instance g, oldest first (the last
// KHIST_LEN iterations): residuals into f, max |dv| into dv; returns the count.
int history_of(const std::vector<double>& hist, int ld, const InstState& s, int g, double* f,
               double* dv) {
  const int m = std::min(s.hist_n, KHIST_LEN);
  for (int j = 0; j < m; ++j) {
    const int k = (s.hist_n - m + j) % KHIST_LEN;
    f[j] = hist[(size_t)(2 * k) * ld + g];
    dv[j] = hist[(size_t)(2 * k + 1) * ld + g];
  }
  return m;
}

// ConvergenceEngine::classifyFailure (solvers/convergence_engine.h:26-87) on
// an instance's DC history: singular > exponential overflow (a step above
// 100 V anywhere in the history) > divergence (the residual rose over each of
// the last 5 iterations) > limit cycle (the residual changed direction in more
// than 60 % of the iterations) > slow convergence (less than a 50 % reduction
// over the last 10). Like the reference, it classifies converged solves too.
// The device keeps the whole-history quantities as running counts, and the
// last KHIST_LEN residuals, which cover the 5- and 10-iteration windows.
int classify_failure(const InstState& s, const double* f, int m) {
  if (s.hflags & KHF_SINGULAR) return KARAM_FAIL_SINGULAR_MATRIX;
  if (s.hist_n == 0) return KARAM_FAIL_NONE;
  if (s.hflags & KHF_OVERFLOW) return KARAM_FAIL_EXPONENTIAL_OVERFLOW;
  if (s.hist_n >= 5) {
    bool rising = true;
    for (int j = m - 4; j < m; ++j)
      if (!(f[j] > f[j - 1])) rising = false;
    if (rising) return KARAM_FAIL_DIVERGENCE;
  }
  if (s.hist_n >= 4 && (double)s.dir_changes / (double)(s.hist_n - 2) > 0.6)
    return KARAM_FAIL_LIMIT_CYCLE;
  if (s.hist_n >= 10) {
    const double first = f[m - 10], last = f[m - 1];
    if (first > 0.0 && last > 0.5 * first) return KARAM_FAIL_SLOW_CONVERGENCE;
  }
  return KARAM_FAIL_NONE;
}

void read_stats(karam_problem* p, karam_instance_stats* stats, bool dc_only) {
  if (!stats) return;
  std::vector<InstState> st(p->ni);
  ck(cudaMemcpy(st.data(), p->i_st.p, st.size() * sizeof(InstState), cudaMemcpyDeviceToHost), "D2H state");
  std::vector<double> hist((size_t)p->ld * 2 * KHIST_LEN);
  ck(cudaMemcpy(hist.data(), p->i_hist.p, hist.size() * sizeof(double), cudaMemcpyDeviceToHost),
     "D2H history");
  for (int i = 0; i < p->ni; ++i) {
    const InstState& s = st[i];
    karam_instance_stats& o = stats[i];
    o.status = s.mode == MODE_DONE ? s.status : KARAM_ST_TIMEOUT;
    o.iterations = dc_only ? s.iters : s.iters + s.tran_iters;
    o.polish_iters = s.polish;
    o.damped = s.damped;
    o.gmin_step = s.g;
    o.seeded_ok = s.seeded_ok;
    o.rescued = s.rescued;
    o.halvings = s.halvings;
    o.max_step_iters = s.max_step_it;
    o.residual = s.resid;
    double f[KHIST_LEN], dv[KHIST_LEN];
    const int m = history_of(hist, p->ld, s, i, f, dv);
    o.failure_type = classify_failure(s, f, m);
    o.stagnation = (s.hflags & KHF_STAGNATION) ? 1 : 0;
    o.divergence = (s.hflags & KHF_DIVERGENCE) ? 1 : 0;
    o.history_len = s.hist_n;
    o.lte_rejects = s.lte_rejects;
  }
}

void read_voltages(karam_problem* p, double* out_v) {
  if (!out_v) return;
  const int n = p->topo.n;
  unpermute(p->i_v.as<double>(), p->t_perm.as<int>(), p->i_out.as<double>(), p->ni, p->ld, n,
            p->ctx->stream);
  ck(cudaMemcpyAsync(out_v, p->i_out.p, (size_t)p->ni * n * sizeof(double), cudaMemcpyDeviceToHost,
                     p->ctx->stream),
     "D2H v");
  ck(cudaStreamSynchronize(p->ctx->stream), "read sync");
}

// Job accounting: counters cleared and a start event recorded before the
// first kernel of a solve call; end_job records the end event and reads back.
void begin_job(karam_problem* p) {
  p->timing = karam_timing{};
  p->seed_timed = false;
  ck(cudaMemsetAsync(p->d_counters.p, 0, 5 * sizeof(unsigned long long), p->ctx->stream), "memset counters");
  ck(cudaEventRecord(p->ev_job0, p->ctx->stream), "event record");
}

void end_job(karam_problem* p) {
  ck(cudaEventRecord(p->ev_job1, p->ctx->stream), "event record");
  unsigned long long c[5];
  ck(cudaMemcpyAsync(c, p->d_counters.p, sizeof(c), cudaMemcpyDeviceToHost, p->ctx->stream), "D2H counters");
  ck(cudaStreamSynchronize(p->ctx->stream), "job sync");
  float ms = 0;
  ck(cudaEventElapsedTime(&ms, p->ev_job0, p->ev_job1), "job time");
  p->timing.job_ms = ms;
  if (p->seed_timed) {
    float sms = 0;
    ck(cudaEventElapsedTime(&sms, p->ev_seed0, p->ev_seed1), "seeder time");
    p->timing.seed_ms = sms;
  }
  p->timing.evals_dc = (int64_t)c[0];
  p->timing.evals_tran = (int64_t)c[1];
  p->timing.solves = (int64_t)c[2];
  p->timing.rescues = (int64_t)c[3];
  p->timing.rescues_dense = (int64_t)c[4];
}

int seeder_features_count(const Topology& T) { return 2 * (int)T.mos.size() + (int)T.vs.size(); }

// KARAM_SEED_MLP: the attached seeder's guess for every instance, written
// instance-interleaved (permuted order) into i_seed.
void mlp_seed(karam_problem* p) {
  karam_seeder* sd = p->seeder;
  if (!sd) throw std::logic_error("KARAM_SEED_MLP without an attached seeder");
  if (karam::mlp_samples(sd->m) == 0) throw std::logic_error("the attached seeder is not trained");
  const int nf = seeder_features_count(p->topo);
  const size_t bytes = (size_t)std::max(1, p->ni) * nf * sizeof(float);
  if (p->i_feat.bytes < bytes) p->i_feat.alloc(bytes);
  cudaStream_t s = p->ctx->stream;
  ck(cudaEventRecord(p->ev_seed0, s), "event record");
  karam::seeder_features(p->dt, dev_inst(p), nullptr, p->ni, p->i_feat.as<float>(), nullptr, s);
  karam::mlp_predict(sd->m, p->i_feat.as<float>(), p->ni, p->i_seed.as<double>(), p->ld, s);
  ck(cudaEventRecord(p->ev_seed1, s), "event record");
  p->seed_timed = true;
  p->timing.other_launches += 1;
}

void start_job(karam_problem* p, const JobParams& P, const double* seed_v) {
  DevInst I = dev_inst(p);
  if (P.seeded == KARAM_SEED_EMA) {
    I.seed = p->i_seed.as<double>();  // written by ema_seed
  } else if (P.seeded == KARAM_SEED_MLP) {
    mlp_seed(p);
    I.seed = p->i_seed.as<double>();
  } else if (P.seeded && seed_v) {
    // caller guesses arrive instance-major in node order; the device works
    // instance-interleaved in permuted order
    const int n = p->topo.n;
    ck(cudaMemcpyAsync(p->i_out.p, seed_v, (size_t)p->ni * n * sizeof(double),
                       cudaMemcpyHostToDevice, p->ctx->stream),
       "H2D seed");
    interleave(p->i_out.as<double>(), p->t_perm.as<int>(), p->i_seed.as<double>(), p->ni, p->ld,
               n, p->ctx->stream);
    p->timing.other_launches += 1;
    I.seed = p->i_seed.as<double>();
  }
  launch_init(p->dt, I, P, p->ctx->stream);
  ck(cudaGetLastError(), "init launch");
  p->timing.other_launches += 1;
  p->tran_started = P.n_steps > 0;
  p->t_now = P.n_steps > 0 ? P.n_steps * P.h : 0.0;
  p->tran_h = P.h;
  p->tran_method = P.method;
}

// KARAM_SEED_EMA: plain DC of the first KARAM_SEED_HISTORY instances, then
// their statistical seed for the whole batch. Returns the parameters of the
// batch job: seeded from lane 0 of i_seed, or plain when the batch is too
// small or the seeder is not confident.
JobParams ema_seed(karam_problem* p, JobParams P, const karam_solver_opts* opts) {
  const int N = p->ni;
  if (N <= KARAM_SEED_HISTORY) {
    P.seeded = KARAM_SEED_NONE;
    return P;
  }
  JobParams P1 = P;
  P1.seeded = KARAM_SEED_NONE;
  P1.n_steps = 0;
  P1.h = 0.0;
  p->ni = KARAM_SEED_HISTORY;
  try {
    start_job(p, P1, nullptr);
    run_rounds(p, P1, opts);
  } catch (...) {
    p->ni = N;
    throw;
  }
  p->ni = N;
  launch_ema_seed(p->dt, dev_inst(p), KARAM_SEED_HISTORY, p->i_seed.as<double>(),
                  p->d_seed_ok.as<int>(), p->ctx->stream);
  ck(cudaGetLastError(), "seed launch");
  p->timing.other_launches += 1;
  ck(cudaMemcpyAsync(p->h_active, p->d_seed_ok.p, sizeof(int), cudaMemcpyDeviceToHost,
                     p->ctx->stream),
     "D2H seed flag");
  ck(cudaStreamSynchronize(p->ctx->stream), "seed sync");
  if (*p->h_active) {
    P.seed_bcast = 1;
  } else {
    P.seeded = KARAM_SEED_NONE;
  }
  return P;
}

}  // namespace

extern "C" {

void karam_default_opts(karam_solver_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = KARAM_PREC_FP64;
  o->max_nr_iter = 50;
  o->gmin_steps = 19;
  o->reltol = 1e-3;
  o->vntol = 1e-6;
  o->kcl_shortcut = 1e-9;
  o->kcl_tol = 1e-12;
  o->polish_max = 0;
  o->polish_rel = 0.0;
  o->polish_abs = 0.0;
  o->lte_reltol = 0.0;
  o->lte_abstol = 0.0;
  o->lu_growth_limit = 0.0;
  o->seeded = 0;
  o->seed_max_iter = 10;
  o->schedule = 0;
  o->max_rounds = 0;
  o->max_halvings = 3;
}

int karam_ctx_create(int device, karam_ctx** out) {
  if (!out) return KARAM_E_INVALID;
  *out = nullptr;
  try {
    int count = 0;
    ck(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    if (device < 0 || device >= count) throw CudaError("no CUDA device with that index");
    ck(cudaSetDevice(device), "cudaSetDevice");
    auto c = std::make_unique<karam_ctx>();
    c->device = device;
    ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device), "attr");
    ck(cudaDeviceGetAttribute(&c->max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device), "attr");
    *out = c.release();
    return KARAM_OK;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    return KARAM_E_CUDA;
  }
}

void karam_ctx_destroy(karam_ctx* ctx) {
  if (!ctx) return;
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* karam_last_error(const karam_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

namespace {

// The netlist's content as bytes (every count, index, value, model name and
// the temperature), the key of the symbolic-analysis cache.
std::string netlist_bytes(const karam_netlist* nl) {
  std::string b;
  auto put = [&](const void* p, size_t n) {
    if (p && n) b.append(static_cast<const char*>(p), n);
    const uint64_t len = n;  // lengths keep distinct layouts distinct
    b.append(reinterpret_cast<const char*>(&len), sizeof(len));
  };
  auto ints = [&](const int32_t* p, int n) { put(p, p ? sizeof(int32_t) * (size_t)n : 0); };
  auto dbls = [&](const double* p, int n) { put(p, p ? sizeof(double) * (size_t)n : 0); };
  put(&nl->n_nodes, sizeof(nl->n_nodes));
  put(&nl->temp_k, sizeof(nl->temp_k));
  const int32_t counts[7] = {nl->n_vsrc, nl->n_isrc, nl->n_res, nl->n_cap, nl->n_dio, nl->n_mos, nl->n_models};
  put(counts, sizeof(counts));
  ints(nl->vs_pos, nl->n_vsrc);
  ints(nl->vs_neg, nl->n_vsrc);
  dbls(nl->vs_dc, nl->n_vsrc);
  ints(nl->vs_kind, nl->n_vsrc);
  dbls(nl->vs_pulse, 7 * nl->n_vsrc);
  ints(nl->is_pos, nl->n_isrc);
  ints(nl->is_neg, nl->n_isrc);
  dbls(nl->is_amp, nl->n_isrc);
  ints(nl->r_n1, nl->n_res);
  ints(nl->r_n2, nl->n_res);
  dbls(nl->r_ohm, nl->n_res);
  ints(nl->c_n1, nl->n_cap);
  ints(nl->c_n2, nl->n_cap);
  dbls(nl->c_farad, nl->n_cap);
  ints(nl->d_anode, nl->n_dio);
  ints(nl->d_cathode, nl->n_dio);
  dbls(nl->d_is, nl->n_dio);
  dbls(nl->d_n, nl->n_dio);
  dbls(nl->d_vt, nl->n_dio);
  ints(nl->d_model, nl->n_dio);
  ints(nl->m_d, nl->n_mos);
  ints(nl->m_g, nl->n_mos);
  ints(nl->m_s, nl->n_mos);
  ints(nl->m_b, nl->n_mos);
  dbls(nl->m_w, nl->n_mos);
  dbls(nl->m_l, nl->n_mos);
  ints(nl->m_model, nl->n_mos);
  ints(nl->model_type, nl->n_models);
  dbls(nl->model_kp, nl->n_models);
  dbls(nl->model_vto, nl->n_models);
  dbls(nl->model_lambda, nl->n_models);
  for (int k = 0; k < nl->n_models; ++k) {
    const char* nm = nl->model_name && nl->model_name[k] ? nl->model_name[k] : "";
    put(nm, std::strlen(nm));
  }
  return b;
}

uint64_t fnv1a(const std::string& b) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : b) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

// Built symbolic analyses by netlist content, most recent first; the role of
// the reference's compiled-block / pattern cache keyed by topologyHash
// (infrastructure/compiled_block.h:45-88, solvers/circuitsim_solver.cpp:262-268).
struct SymbolicCache {
  static constexpr size_t kEntries = 32;
  static constexpr size_t kBytes = size_t(8) << 30;  // tables kept across entries
  struct Entry {
    std::string key;
    std::shared_ptr<const Topology> topo;
    size_t bytes;
  };
  std::mutex mu;
  std::list<Entry> lru;
  size_t bytes = 0;
  int64_t hits = 0, misses = 0;
};

// Host bytes of a built analysis, counted over the tables that grow with the
// fill and the level schedule (the rest is linear in the netlist): several GB
// for a 256 x 256 mesh tile.
size_t topology_bytes(const Topology& T) {
  size_t b = T.trip.size() * sizeof(Triplet);
  for (const std::vector<int>* v :
       {&T.f_col, &T.f_slot, &T.slot_row, &T.slot_col, &T.jt_code, &T.lu_data, &T.lu_rec, &T.nd_src,
        &T.l_slot, &T.l_piv, &T.t_slot, &T.t_off, &T.pr_l, &T.pr_u, &T.y_row, &T.y_off, &T.yp_l, &T.yp_k,
        &T.bs_u, &T.bs_c, &T.nd_prog, &T.es_item, &T.es_jt, &T.es_ft})
    b += v->size() * sizeof(int);
  return b;
}
SymbolicCache& symbolic_cache() {
  static SymbolicCache c;
  return c;
}

Topology cached_topology(const karam_netlist* nl) {
  const std::string key = netlist_bytes(nl);
  SymbolicCache& C = symbolic_cache();
  {
    std::lock_guard<std::mutex> lock(C.mu);
    for (auto it = C.lru.begin(); it != C.lru.end(); ++it)
      if (it->key == key) {
        C.lru.splice(C.lru.begin(), C.lru, it);
        ++C.hits;
        return *C.lru.front().topo;
      }
    ++C.misses;
  }
  auto T = std::make_shared<const Topology>(build_topology(nl));  // outside the lock
  const size_t tb = topology_bytes(*T);
  if (tb > SymbolicCache::kBytes) return *T;  // larger than the whole budget: not kept
  std::lock_guard<std::mutex> lock(C.mu);
  for (const auto& e : C.lru)
    if (e.key == key) return *T;  // another thread kept the same analysis meanwhile
  C.lru.push_front({key, T, tb});
  C.bytes += tb;
  while (C.lru.size() > SymbolicCache::kEntries || C.bytes > SymbolicCache::kBytes) {
    C.bytes -= C.lru.back().bytes;
    C.lru.pop_back();
  }
  return *T;
}

}  // namespace

int karam_netlist_hash(const karam_netlist* nl, uint64_t* out) {
  if (!nl || !out) return KARAM_E_INVALID;
  *out = fnv1a(netlist_bytes(nl));
  return KARAM_OK;
}

int karam_symbolic_cache_info(int32_t* entries, int64_t* hits, int64_t* misses) {
  SymbolicCache& C = symbolic_cache();
  std::lock_guard<std::mutex> lock(C.mu);
  if (entries) *entries = (int32_t)C.lru.size();
  if (hits) *hits = C.hits;
  if (misses) *misses = C.misses;
  return KARAM_OK;
}

void karam_symbolic_cache_clear(void) {
  SymbolicCache& C = symbolic_cache();
  std::lock_guard<std::mutex> lock(C.mu);
  C.lru.clear();
  C.bytes = 0;
  C.hits = C.misses = 0;
}

int karam_problem_create(karam_ctx* ctx, const karam_netlist* nl, int32_t max_instances,
                         karam_problem** out) {
  if (!out) return KARAM_E_INVALID;
  *out = nullptr;
  return guarded(ctx, [&] {
    if (max_instances < 1) throw std::runtime_error("max_instances must be >= 1");
    if (!nl) throw std::runtime_error("no netlist");
    auto p = std::make_unique<karam_problem>();
    p->topo = cached_topology(nl);
    p->content_hash = fnv1a(netlist_bytes(nl));
    p->max_inst = max_instances;
    if (!ctx) {  // symbolic analysis only
      *out = p.release();
      return KARAM_OK;
    }
    ck(cudaSetDevice(ctx->device), "cudaSetDevice");
    p->ctx = ctx;
    upload_topology(p.get());
    alloc_instances(p.get());
    set_instances_impl(p.get(), nullptr);
    *out = p.release();
    return KARAM_OK;
  });
}

void karam_problem_destroy(karam_problem* p) { delete p; }

int karam_problem_info_get(const karam_problem* p, karam_problem_info* o) {
  if (!p || !o) return KARAM_E_INVALID;
  const Topology& T = p->topo;
  o->n = T.n;
  o->nnz = T.nnz();
  o->nnz_filled = T.nnz_filled();
  o->fill_in = T.fill_in;
  o->treewidth = T.treewidth;
  o->n_triplets = (int)T.trip.size();
  o->n_instances = p->ni;
  o->n_mos = (int)T.mos.size();
  o->n_dio = (int)T.dio.size();
  o->n_res = (int)T.res.size();
  o->n_cap = (int)T.cap.size();
  o->n_vsrc = (int)T.vs.size();
  o->n_isrc = (int)T.isrc.size();
  o->lu_ops = T.lu_ops;
  o->n_slots = T.nv;
  o->es_blocks = (int32_t)T.es_block.size() / 4;
  o->es_device_evals = (int32_t)T.es_dev.size();
  return KARAM_OK;
}

int karam_set_instances(karam_problem* p, const karam_instances* inst) {
  if (!p) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    set_instances_impl(p, inst);
    return KARAM_OK;
  });
}

int karam_solve_dc(karam_problem* p, const karam_solver_opts* opts, const double* seed_v,
                   double* out_v, karam_instance_stats* stats) {
  if (!p) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    JobParams P = job_params(opts, 0, 0.0, KARAM_TRAN_BE);
    if (P.seeded == KARAM_SEED_CALLER && !seed_v)
      throw std::runtime_error("seeded solve without seed_v");
    begin_job(p);
    if (P.seeded == KARAM_SEED_EMA) P = ema_seed(p, P, opts);
    start_job(p, P, seed_v);
    run_rounds(p, P, opts);
    end_job(p);
    p->have_dc = true;
    read_voltages(p, out_v);
    read_stats(p, stats, true);
    return KARAM_OK;
  });
}

int karam_run_mc_device(karam_problem* p, const karam_solver_opts* opts, double dt,
                        int32_t n_steps, int32_t method) {
  if (!p) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    JobParams P = job_params(opts, n_steps, dt, method);
    if (P.seeded == KARAM_SEED_CALLER)
      throw std::runtime_error("caller seeds need karam_solve_dc");
    begin_job(p);
    if (P.seeded == KARAM_SEED_EMA) P = ema_seed(p, P, opts);
    start_job(p, P, nullptr);
    run_rounds(p, P, opts);
    end_job(p);
    p->have_dc = true;
    return KARAM_OK;
  });
}

int karam_run_mc_multi(karam_problem* const* probs, int32_t n_probs, const karam_solver_opts* opts,
                       double dt, int32_t n_steps, int32_t method) {
  if (!probs || n_probs < 1) return KARAM_E_INVALID;
  for (int j = 0; j < n_probs; ++j)
    if (!probs[j] || probs[j]->ctx != probs[0]->ctx) return KARAM_E_INVALID;
  {  // each problem once: its buffers are its instances' state for the launch
    std::vector<const karam_problem*> seen(probs, probs + n_probs);
    std::sort(seen.begin(), seen.end());
    if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) return KARAM_E_INVALID;
  }
  karam_ctx* ctx = probs[0]->ctx;
  return guarded(ctx, [&] {
    for (int j = 0; j < n_probs; ++j) need_device(probs[j]);
    const JobParams P = job_params(opts, n_steps, dt, method);
    if (P.seeded != KARAM_SEED_NONE) throw std::runtime_error("karam_run_mc_multi runs unseeded jobs only");
    const int prec = P.precision;
    cudaStream_t s = ctx->stream;
    // one table entry per problem, CTA ranges back to back, the costliest
    // instances (most LU operations per factorisation) first: CTAs start in
    // index order, so the longest ones do not trail the launch
    std::vector<int> order(n_probs);
    for (int j = 0; j < n_probs; ++j) order[j] = j;
    auto cost = [&](int j) { return (double)probs[j]->topo.lu_ops + (double)probs[j]->topo.nnz(); };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<PersistJob> jobs(n_probs);
    std::vector<size_t> lock_off(n_probs);
    std::vector<char> resident(n_probs, 0);
    size_t smem = 16, n_locks = 0;
    int grid = 0;
    for (int q = 0; q < n_probs; ++q) {
      const int j = order[q];
      karam_problem* p = probs[j];
      const PersistPlan plan = plan_persist_job(p->dt, prec, p->rplan, ctx->max_smem);
      cudaGetLastError();
      if (plan.smem == 0 || p->max_hub_chunks > 8)
        throw std::runtime_error("problem " + std::to_string(j) +
                                 " does not fit the multi-problem persistent kernel");
      PersistJob& J = jobs[q];
      std::memset(&J, 0, sizeof(J));
      J.T = p->dt;
      J.I = dev_inst(p);
      J.P = P;
      J.K = p->rplan.K;
      J.I.rescue_list = nullptr;  // no hand-off: a solve with no rescue slot is singular
      J.cta0 = grid;
      J.variant = plan.variant;
      J.resident_at = plan.resident_at;
      J.slot_values = plan.slot_values;
      resident[j] = plan.resident_at > 0;
      lock_off[q] = n_locks;
      n_locks += p->rescue_slots;
      if (plan.variant == 2) {
        const size_t need = (size_t)p->ni * (size_t)p->dt.nd_S * sizeof(double);
        if (p->i_luws.bytes < need) p->i_luws.alloc(need);
        J.I.lu_ws = p->i_luws.p;
      }
      smem = std::max(smem, plan.smem);
      grid += p->ni;
    }
    // [active, rounds_max, slot timeouts, pad, slot locks...]
    DBuf words;
    words.alloc((4 + n_locks) * sizeof(int));
    int* d_words = words.as<int>();
    for (int j = 0; j < n_probs; ++j) jobs[j].slot_lock = d_words + 4 + lock_off[j];
    DBuf table;
    upload(table, jobs);
    ck(cudaMemsetAsync(d_words, 0, words.bytes, s), "memset launch words");
    for (int j = 0; j < n_probs; ++j) begin_job(probs[j]);
    for (int j = 0; j < n_probs; ++j) start_job(probs[j], P, nullptr);
    if (grid > 0) {
      const int budget = opts && opts->max_rounds > 0 ? opts->max_rounds : (1 << 30);
      launch_persist_multi(table.as<PersistJob>(), n_probs, prec, grid, smem, budget, d_words,
                           d_words + 1, d_words + 2, s);
      ck(cudaGetLastError(), "k_persist_multi launch");
    }
    int h_words[4] = {0, 0, 0, 0};
    ck(cudaMemcpyAsync(h_words, d_words, sizeof(h_words), cudaMemcpyDeviceToHost, s), "D2H active");
    ck(cudaStreamSynchronize(s), "persistent sync");
    for (int j = 0; j < n_probs; ++j) {
      karam_problem* p = probs[j];
      p->timing.lanes = 1;
      p->timing.level_schedule = 5;
      p->timing.rounds = h_words[1];
      p->timing.persistent_rounds = h_words[1];
      p->timing.resident_instances = resident[j] ? p->ni : 0;
      p->timing.other_launches += j == 0 ? 1 : 0;
      end_job(p);
      p->have_dc = true;
    }
    if (h_words[2] > 0)
      throw CudaError(std::to_string(h_words[2]) +
                      " solves found no free rescue workspace slot in time; their instances "
                      "report KARAM_ST_SINGULAR");
    return KARAM_OK;
  });
}

int karam_tune_schedule(karam_problem* p, const karam_solver_opts* opts, int32_t rounds,
                        int32_t* schedule, double* best_ms) {
  if (!p || rounds < 1) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    karam_solver_opts o;
    if (opts)
      o = *opts;
    else
      karam_default_opts(&o);
    o.max_rounds = rounds;
    o.kernel_timing = 0;
    o.seeded = KARAM_SEED_NONE;  // trial rounds from the reference seed
    const int prec = o.precision;
    // the feasible schedules: the planner's choice, then a CTA per instance
    // with the slots and the packed program in shared memory, with the slots
    // alone in shared memory, or in global memory (option values as in
    // karam_solver_opts.schedule)
    std::vector<int> cands;
    for (int want : {0, -3, -1, -2}) {
      const RoundLaunch L = plan_round(p->dt, p->ni, prec, p->ctx->max_smem, p->ctx->num_sms, want);
      cudaGetLastError();
      if (L.L < 1) continue;
      const int val = L.big ? -L.big : L.L;
      if (std::find(cands.begin(), cands.end(), val) == cands.end()) cands.push_back(val);
    }
    if (p->max_hub_chunks <= 8 && (p->rescue_slots == 0 || p->rescue_slots >= p->ni) &&
        plan_persist(p->dt, prec, p->rplan, p->ctx->max_smem).smem > 0)
      cands.push_back(-4);
    cudaGetLastError();
    if (cands.empty()) throw std::runtime_error("no factor/solve schedule fits this problem");
    int best = cands[0];
    double best_t = 1e300;
    for (int c : cands) {
      o.schedule = c;
      const JobParams P = job_params(&o, 0, 0.0, KARAM_TRAN_BE);
      double t = 1e300;
      for (int rep = 0; rep < 2; ++rep) {  // the first trial builds the graph
        begin_job(p);
        start_job(p, P, nullptr);
        run_rounds(p, P, &o);
        end_job(p);
        t = std::min(t, p->timing.job_ms);
      }
      if (t < best_t) {
        best_t = t;
        best = c;
      }
    }
    p->tuned[prec == KARAM_PREC_MIXED ? 1 : 0] = best;
    {
      std::lock_guard<std::mutex> lock(g_tune_mu);
      tune_cache()[tune_key(p, prec)] = best;
    }
    p->have_dc = false;  // the state is a trial's
    if (schedule) *schedule = best;
    if (best_ms) *best_ms = best_t;
    return KARAM_OK;
  });
}

int karam_get_history(karam_problem* p, int32_t instance, double* residual, double* max_dv,
                      int32_t* len) {
  if (!p || !len || (!residual) != (!max_dv)) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    if (instance < 0 || instance >= p->ni) throw std::runtime_error("instance out of range");
    ck(cudaStreamSynchronize(p->ctx->stream), "sync");
    InstState s;
    ck(cudaMemcpy(&s, p->i_st.as<InstState>() + instance, sizeof(s), cudaMemcpyDeviceToHost),
       "D2H state");
    std::vector<double> hist((size_t)p->ld * 2 * KHIST_LEN);
    ck(cudaMemcpy(hist.data(), p->i_hist.p, hist.size() * sizeof(double), cudaMemcpyDeviceToHost),
       "D2H history");
    double f[KHIST_LEN], dv[KHIST_LEN];
    const int m = history_of(hist, p->ld, s, instance, f, dv);
    *len = m;
    if (residual)
      for (int j = 0; j < m; ++j) {
        residual[j] = f[j];
        max_dv[j] = dv[j];
      }
    return KARAM_OK;
  });
}

int karam_read_results(karam_problem* p, double* out_v, karam_instance_stats* stats) {
  if (!p) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    read_voltages(p, out_v);
    read_stats(p, stats, false);
    return KARAM_OK;
  });
}

int karam_run_mc(karam_problem* p, const karam_instances* inst, const karam_solver_opts* opts,
                 double dt, int32_t n_steps, int32_t method, double* out_v,
                 karam_instance_stats* stats) {
  if (!p) return KARAM_E_INVALID;
  int rc = karam_set_instances(p, inst);
  if (rc != KARAM_OK) return rc;
  rc = karam_run_mc_device(p, opts, dt, n_steps, method);
  if (rc != KARAM_OK) return rc;
  return karam_read_results(p, out_v, stats);
}

int karam_step_transient(karam_problem* p, const karam_solver_opts* opts, double dt,
                         int32_t n_steps, int32_t method, const int32_t* wave_nodes,
                         int32_t n_wave, double* wave_out, double* out_v,
                         karam_instance_stats* stats) {
  if (!p) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    if (!p->have_dc) throw std::runtime_error("karam_step_transient needs a DC solution first");
    if (n_steps < 1) throw std::runtime_error("n_steps must be >= 1");
    if (n_wave > 0 && (!wave_nodes || !wave_out)) throw std::runtime_error("wave buffers missing");
    if (p->tran_started && (dt != p->tran_h || method != p->tran_method))
      throw std::runtime_error("a transient continues with the step and method it started with");
    JobParams P = job_params(opts, n_steps, dt, method);
    P.t0 = p->t_now;
    DevInst I = dev_inst(p);
    DBuf wave, wpos;
    if (n_wave > 0) {
      std::vector<int> pos(n_wave);
      for (int k = 0; k < n_wave; ++k) {
        int node = wave_nodes[k];
        if (node < 0 || node > p->topo.n) throw std::runtime_error("wave node out of range");
        pos[k] = node > 0 ? p->topo.iperm[node - 1] : -1;
      }
      upload(wpos, pos);
      wave.alloc((size_t)p->ni * n_steps * n_wave * sizeof(double));
      ck(cudaMemset(wave.p, 0, wave.bytes), "memset wave");
    }
    I.wave = wave.as<double>();
    I.wave_pos = wpos.as<int>();
    I.n_wave = n_wave;
    I.wave_steps = n_steps;
    begin_job(p);
    launch_tran_start(p->dt, I, P, p->tran_started ? 0 : 1, p->ctx->stream);
    ck(cudaGetLastError(), "tran start");
    p->timing.other_launches += 1;
    run_rounds(p, P, opts, &I);
    end_job(p);
    p->tran_started = true;
    p->tran_h = dt;
    p->tran_method = method;
    p->t_now += n_steps * dt;
    if (n_wave > 0)
      ck(cudaMemcpy(wave_out, wave.p, wave.bytes, cudaMemcpyDeviceToHost), "D2H wave");
    read_voltages(p, out_v);
    read_stats(p, stats, false);
    return KARAM_OK;
  });
}

int karam_sync(karam_problem* p) {
  if (!p) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    ck(cudaStreamSynchronize(p->ctx->stream), "sync");
    return KARAM_OK;
  });
}

int karam_get_pattern(const karam_problem* p, int32_t* row_ptr, int32_t* col) {
  if (!p) return KARAM_E_INVALID;
  if (row_ptr) std::copy(p->topo.row_ptr.begin(), p->topo.row_ptr.end(), row_ptr);
  if (col) std::copy(p->topo.col.begin(), p->topo.col.end(), col);
  return KARAM_OK;
}

int karam_get_stamp_map(const karam_problem* p, int32_t* slot_csr) {
  if (!p || !slot_csr) return KARAM_E_INVALID;
  std::copy(p->topo.slot_csr.begin(), p->topo.slot_csr.end(), slot_csr);
  return KARAM_OK;
}

int karam_get_ordering(const karam_problem* p, uint32_t* raw, int32_t* raw_len, int32_t* perm) {
  if (!p) return KARAM_E_INVALID;
  if (raw) std::copy(p->topo.raw_order.begin(), p->topo.raw_order.end(), raw);
  if (raw_len) *raw_len = (int32_t)p->topo.raw_order.size();
  if (perm) std::copy(p->topo.perm.begin(), p->topo.perm.end(), perm);
  return KARAM_OK;
}

int karam_get_filled_pattern(const karam_problem* p, int32_t* f_row_ptr, int32_t* f_col) {
  if (!p) return KARAM_E_INVALID;
  if (f_row_ptr) std::copy(p->topo.f_row_ptr.begin(), p->topo.f_row_ptr.end(), f_row_ptr);
  if (f_col) std::copy(p->topo.f_col.begin(), p->topo.f_col.end(), f_col);
  return KARAM_OK;
}

int karam_get_device_order(const karam_problem* p, int32_t* mos_order, int32_t* dio_order) {
  if (!p) return KARAM_E_INVALID;
  if (mos_order) std::copy(p->topo.mos_order.begin(), p->topo.mos_order.end(), mos_order);
  if (dio_order) std::copy(p->topo.dio_order.begin(), p->topo.dio_order.end(), dio_order);
  return KARAM_OK;
}

int karam_get_lu_program(const karam_problem* p, int32_t* hdr, int32_t* data, int32_t* data_len,
                         int32_t* slot_rc) {
  if (!p) return KARAM_E_INVALID;
  const Topology& T = p->topo;
  if (hdr) std::copy(T.lu_hdr.begin(), T.lu_hdr.end(), hdr);
  if (data_len) *data_len = (int32_t)T.lu_data.size();
  if (data) std::copy(T.lu_data.begin(), T.lu_data.end(), data);
  if (slot_rc)
    for (int s = 0; s < T.nv; ++s) {
      slot_rc[2 * s] = T.slot_row[s];
      slot_rc[2 * s + 1] = T.slot_col[s];
    }
  return KARAM_OK;
}

int karam_get_lu_records(const karam_problem* p, int32_t* rec, int32_t* rec2) {
  if (!p) return KARAM_E_INVALID;
  const Topology& T = p->topo;
  if (!T.lu_small) return KARAM_E_UNSUPPORTED;
  if (rec) std::copy(T.lu_rec.begin(), T.lu_rec.end(), rec);
  if (rec2) std::copy(T.lu_rec2.begin(), T.lu_rec2.end(), rec2);
  return KARAM_OK;
}

int karam_get_lu_schedule(const karam_problem* p, int32_t* buf, int64_t cap, int64_t* len) {
  if (!p || !len) return KARAM_E_INVALID;
  const Topology& T = p->topo;
  if (T.nd_levels == 0) return KARAM_E_UNSUPPORTED;
  std::vector<int32_t> out{T.n, T.nd_nv, T.nd_levels, Topology::kNdLong};
  for (const std::vector<int>* v :
       {&T.nd_perm, &T.nd_src, &T.nd_diag, &T.lv_piv, &T.lv_piv_ptr, &T.lv_l_ptr, &T.l_slot,
        &T.l_piv, &T.lv_ts_ptr, &T.lv_tl_ptr, &T.t_slot, &T.t_off, &T.pr_l, &T.pr_u, &T.lv_ys_ptr,
        &T.lv_yl_ptr, &T.y_row, &T.y_off, &T.yp_l, &T.yp_k, &T.bs_off, &T.bs_u, &T.bs_c,
        &T.nd_prog}) {
    out.push_back((int32_t)v->size());
    out.insert(out.end(), v->begin(), v->end());
  }
  *len = (int64_t)out.size();
  if (buf && cap >= (int64_t)out.size()) std::copy(out.begin(), out.end(), buf);
  return KARAM_OK;
}

int karam_ac_sweep(karam_problem* p, double f_start, double f_stop, int32_t n_points,
                   int32_t input_node, double amplitude, double* freqs_out, double* out_re,
                   double* out_im, int32_t* status) {
  if (!p || n_points < 1 || !out_re || !out_im) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    if (!p->have_dc || p->tran_started)
      throw std::logic_error("karam_ac_sweep needs a DC operating point (a DC-only solve first)");
    const Topology& T = p->topo;
    const int n = T.n, ni = p->ni;
    const size_t ld = (size_t)p->ld;
    if (input_node < 0 || input_node > n) throw std::runtime_error("input node out of range");
    int stage = 0;
    const size_t smem = plan_ac(p->dt, p->ctx->max_smem, &stage);
    cudaGetLastError();
    if (smem == 0) {
      set_err(p->ctx, "AC needs the packed level program and its complex slots in one CTA's shared memory");
      return KARAM_E_UNSUPPORTED;
    }
    // log-spaced frequencies, ACSolver::solveAC_Sparse's formula (ac_solver.h:724-729)
    std::vector<double> f(n_points), w(n_points);
    const double lo = std::log10(std::max(f_start, 1e-3));
    const double hi = std::log10(std::max(f_stop, f_start + 1.0));
    for (int k = 0; k < n_points; ++k) {
      f[k] = std::pow(10.0, lo + (hi - lo) * k / std::max(n_points - 1, 1));
      w[k] = 2.0 * M_PI * f[k];
    }
    if (freqs_out) std::copy(f.begin(), f.end(), freqs_out);
    cudaStream_t s = p->ctx->stream;
    // the FP64 Jacobian of every instance at its DC point
    ck(cudaMemcpyAsync(p->i_x.p, p->i_v.p, (size_t)n * ld * sizeof(double), cudaMemcpyDeviceToDevice, s),
       "copy v");
    std::vector<double> evh(ld, -1.0), evt(ld, 0.0);
    std::fill(evh.begin(), evh.begin() + ni, 0.0);
    ck(cudaMemcpyAsync(p->i_evh.p, evh.data(), ld * sizeof(double), cudaMemcpyHostToDevice, s), "H2D ev");
    ck(cudaMemcpyAsync(p->i_evt.p, evt.data(), ld * sizeof(double), cudaMemcpyHostToDevice, s), "H2D ev");
    JobParams P = job_params(nullptr, 0, 0.0, KARAM_TRAN_BE);
    P.precision = KARAM_PREC_FP64;
    DevInst I = dev_inst(p);
    const RoundLaunch L = plan_round(p->dt, ni, KARAM_PREC_FP64, p->ctx->max_smem, p->ctx->num_sms, 0);
    if (L.L < 1) throw std::runtime_error(std::string("no evaluation schedule fits: ") + L.why);
    DBuf d_w, d_re, d_im, d_st;
    d_w.alloc((size_t)n_points * sizeof(double));
    const size_t npts = (size_t)ni * n_points;
    d_re.alloc(npts * n * sizeof(double));
    d_im.alloc(npts * n * sizeof(double));
    d_st.alloc(npts * sizeof(int));
    ck(cudaMemcpyAsync(d_w.p, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice, s), "H2D omega");
    p->timing = karam_timing{};
    ck(cudaEventRecord(p->ev_job0, s), "event record");
    launch_eval_stamp(p->dt, I, P, L, KARAM_PREC_FP64, s);
    ck(cudaGetLastError(), "eval launch");
    AcParams A{};
    A.omega = d_w.as<double>();
    A.n_points = n_points;
    A.in_pos = input_node > 0 ? T.iperm[input_node - 1] : -1;
    A.in_slot = A.in_pos >= 0 ? T.lu_hdr[4 * A.in_pos + 3] : -1;
    A.stage_prog = stage;
    A.g_in = 1e6;  // the excitation's Norton conductance (ac_solver.h:751-763)
    A.rhs_in = 1e6 * amplitude;
    A.gmin = 1e-12;
    A.tiny = 1e-25;
    A.growth = P.growth64;
    A.perm = p->t_perm.as<int>();
    A.out_re = d_re.as<double>();
    A.out_im = d_im.as<double>();
    A.status = d_st.as<int>();
    launch_ac(p->dt, I, A, smem, s);
    ck(cudaGetLastError(), "k_ac launch");
    ck(cudaEventRecord(p->ev_job1, s), "event record");
    ck(cudaMemcpyAsync(out_re, d_re.p, npts * n * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H ac");
    ck(cudaMemcpyAsync(out_im, d_im.p, npts * n * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H ac");
    std::vector<int> st_ac(npts);
    ck(cudaMemcpyAsync(st_ac.data(), d_st.p, npts * sizeof(int), cudaMemcpyDeviceToHost, s), "D2H status");
    std::vector<InstState> st(ni);
    ck(cudaMemcpyAsync(st.data(), p->i_st.p, ni * sizeof(InstState), cudaMemcpyDeviceToHost, s), "D2H state");
    // every instance's evaluation point back to "done"
    std::fill(evh.begin(), evh.end(), -1.0);
    ck(cudaMemcpyAsync(p->i_evh.p, evh.data(), ld * sizeof(double), cudaMemcpyHostToDevice, s), "H2D ev");
    ck(cudaStreamSynchronize(s), "ac sync");
    float ms = 0;
    ck(cudaEventElapsedTime(&ms, p->ev_job0, p->ev_job1), "ac time");
    p->timing.job_ms = ms;
    p->timing.eval_launches = 1;
    p->timing.other_launches = 1;
    if (status)
      for (int g = 0; g < ni; ++g) {
        // an instance whose DC point did not converge reports that status
        const int dc = st[g].mode == MODE_DONE ? st[g].status : KARAM_ST_TIMEOUT;
        for (int k = 0; k < n_points; ++k)
          status[(size_t)g * n_points + k] = dc != KARAM_ST_CONVERGED ? dc : st_ac[(size_t)g * n_points + k];
      }
    return KARAM_OK;
  });
}

int karam_eval_stamp(karam_problem* p, int32_t precision, const double* v, double* jac, double* f) {
  if (!p || !v) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    if (precision != KARAM_PREC_FP64 && precision != KARAM_PREC_MIXED)
      throw std::runtime_error("unknown precision");
    const Topology& T = p->topo;
    const int n = T.n, nvs = T.nv, ni = p->ni;
    const size_t ld = (size_t)p->ld;
    cudaStream_t s = p->ctx->stream;
    ck(cudaMemcpyAsync(p->i_out.p, v, (size_t)ni * n * sizeof(double), cudaMemcpyHostToDevice, s), "H2D v");
    interleave(p->i_out.as<double>(), p->t_perm.as<int>(), p->i_x.as<double>(), ni, p->ld, n, s);
    // every instance evaluates a DC point
    std::vector<double> evh(ld, -1.0), evt(ld, 0.0);
    std::fill(evh.begin(), evh.begin() + ni, 0.0);
    ck(cudaMemcpyAsync(p->i_evh.p, evh.data(), ld * sizeof(double), cudaMemcpyHostToDevice, s), "H2D ev");
    ck(cudaMemcpyAsync(p->i_evt.p, evt.data(), ld * sizeof(double), cudaMemcpyHostToDevice, s), "H2D ev");
    JobParams P = job_params(nullptr, 0, 0.0, KARAM_TRAN_BE);
    P.precision = precision;
    DevInst I = dev_inst(p);
    const RoundLaunch L = plan_round(p->dt, ni, precision, p->ctx->max_smem, p->ctx->num_sms, 0);
    p->timing = karam_timing{};
    ck(cudaEventRecord(p->ev_job0, s), "event record");
    launch_eval_stamp(p->dt, I, P, L, precision, s);
    ck(cudaGetLastError(), "eval launch");
    ck(cudaEventRecord(p->ev_job1, s), "event record");
    std::vector<double> F((size_t)n * ld);
    ck(cudaMemcpyAsync(F.data(), p->i_F.p, F.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H F");
    std::vector<double> J64;
    std::vector<float> J32;
    if (precision == KARAM_PREC_MIXED) {
      J32.resize((size_t)nvs * ld);
      ck(cudaMemcpyAsync(J32.data(), p->i_J.p, J32.size() * sizeof(float), cudaMemcpyDeviceToHost, s), "D2H J");
    } else {
      J64.resize((size_t)nvs * ld);
      ck(cudaMemcpyAsync(J64.data(), p->i_J.p, J64.size() * sizeof(double), cudaMemcpyDeviceToHost, s), "D2H J");
    }
    ck(cudaStreamSynchronize(s), "eval sync");
    float ms = 0;
    ck(cudaEventElapsedTime(&ms, p->ev_job0, p->ev_job1), "eval time");
    p->timing.job_ms = p->timing.eval_ms = ms;
    p->timing.eval_launches = 1;
    p->timing.other_launches = 1;  // the interleave of the caller's voltages
    // the device state no longer holds a solution
    p->have_dc = false;
    std::vector<double> neg(ld, -1.0);
    ck(cudaMemcpy(p->i_evh.p, neg.data(), ld * sizeof(double), cudaMemcpyHostToDevice), "reset ev");
    const int nnz = T.nnz();
    for (int i = 0; i < ni; ++i) {
      if (jac)
        for (int j = 0; j < nnz; ++j) {
          const int sl = p->csr_to_slot[j];
          double val = 0.0;
          if (sl >= 0) {
            const size_t src = (size_t)sl * ld + i;
            val = precision == KARAM_PREC_MIXED ? (double)J32[src] : J64[src];
          }
          jac[(size_t)i * nnz + j] = val;
        }
      if (f)
        for (int k = 0; k < n; ++k) f[(size_t)i * n + T.perm[k]] = F[(size_t)k * ld + i];
    }
    return KARAM_OK;
  });
}

int karam_eval_stamp_noalloc(karam_problem* p, int32_t precision, const double* d_v,
                             double* d_jac, double* d_f) {
  if (!p || !d_v || !d_jac || !d_f) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    if (precision != KARAM_PREC_FP64 && precision != KARAM_PREC_MIXED)
      throw std::runtime_error("unknown precision");
    const Topology& T = p->topo;
    const size_t need = noalloc_bytes(T.n, T.nv, T.nnz(), p->ld, T.n_hub_rows, T.n_hub_groups);
    if (need > kScratchBytes)
      throw std::runtime_error("karam_eval_stamp_noalloc: this problem needs " +
                               std::to_string(need) + " bytes of scratch, the fixed maximum is " +
                               std::to_string(kScratchBytes) +
                               " (create the problem with fewer max_instances)");
    ck(cudaSetDevice(p->ctx->device), "cudaSetDevice");
    const char* err = "";
    void* scratch = noalloc_scratch(&err);
    if (!scratch) throw CudaError(std::string("cudaGetSymbolAddress: ") + err);
    cudaStream_t s = p->ctx->stream;
    ck(noalloc_eval_stamp(scratch, p->dt, dev_inst(p), precision, d_v, p->t_perm.as<int>(),
                          p->csr_to_slot.data(), T.nnz(), d_jac, d_f, s),
       "karam_eval_stamp_noalloc launch");
    ck(cudaStreamSynchronize(s), "karam_eval_stamp_noalloc sync");
    return KARAM_OK;
  });
}

int karam_seeder_create(karam_problem* p, int32_t width, int32_t hidden_layers,
                        uint64_t init_seed, karam_seeder** out) {
  if (!p || !out) return KARAM_E_INVALID;
  *out = nullptr;
  return guarded(p->ctx, [&] {
    need_device(p);
    if (width < 1 || width > 8192 || hidden_layers < 0 || hidden_layers > 16)
      throw std::runtime_error("seeder: width must be in 1..8192 and hidden_layers in 0..16");
    const Topology& T = p->topo;
    auto sd = std::make_unique<karam_seeder>();
    sd->ctx = p->ctx;
    sd->n = T.n;
    sd->nv = T.nv;
    sd->n_mos = (int)T.mos.size();
    sd->n_vs = (int)T.vs.size();
    sd->m = karam::mlp_create(seeder_features_count(T), T.n, width, hidden_layers, init_seed,
                              p->ctx->stream);
    *out = sd.release();
    return KARAM_OK;
  });
}

void karam_seeder_destroy(karam_seeder* s) { delete s; }

namespace {
void seeder_matches(const karam_seeder* s, const karam_problem* p) {
  const Topology& T = p->topo;
  if (s->ctx != p->ctx || s->n != T.n || s->nv != T.nv || s->n_mos != (int)T.mos.size() ||
      s->n_vs != (int)T.vs.size())
    throw std::runtime_error("seeder and problem differ in context or topology sizes");
}
}  // namespace

int karam_seeder_add_dc(karam_seeder* s, karam_problem* p, int32_t* added) {
  if (!s || !p) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    seeder_matches(s, p);
    if (!p->have_dc || p->tran_started)
      throw std::logic_error("karam_seeder_add_dc needs a DC solve as the problem's last solve");
    std::vector<InstState> st(p->ni);
    ck(cudaMemcpy(st.data(), p->i_st.p, st.size() * sizeof(InstState), cudaMemcpyDeviceToHost),
       "D2H state");
    std::vector<int> idx;
    for (int g = 0; g < p->ni; ++g)
      if (st[g].status == KST_CONVERGED) idx.push_back(g);
    if (added) *added = (int32_t)idx.size();
    if (idx.empty()) return KARAM_OK;
    const int nf = seeder_features_count(p->topo), rows = (int)idx.size();
    DBuf d_idx, X, Y;
    d_idx.alloc(idx.size() * sizeof(int));
    X.alloc((size_t)rows * nf * sizeof(float));
    Y.alloc((size_t)rows * p->topo.n * sizeof(float));
    cudaStream_t cs = p->ctx->stream;
    ck(cudaMemcpyAsync(d_idx.p, idx.data(), idx.size() * sizeof(int), cudaMemcpyHostToDevice, cs),
       "H2D index");
    karam::seeder_features(p->dt, dev_inst(p), d_idx.as<int>(), rows, X.as<float>(), Y.as<float>(),
                           cs);
    karam::mlp_add_samples(s->m, X.as<float>(), Y.as<float>(), rows, cs);
    ck(cudaStreamSynchronize(cs), "seeder sync");
    return KARAM_OK;
  });
}

int karam_seeder_train(karam_seeder* s, int32_t epochs, int32_t batch, float lr,
                       uint64_t shuffle_seed, float* final_loss) {
  if (!s) return KARAM_E_INVALID;
  return guarded(s->ctx, [&] {
    ck(cudaSetDevice(s->ctx->device), "cudaSetDevice");
    const float l = karam::mlp_train(s->m, epochs, batch, lr, shuffle_seed, s->ctx->stream);
    if (final_loss) *final_loss = l;
    return KARAM_OK;
  });
}

int karam_problem_set_seeder(karam_problem* p, karam_seeder* s) {
  if (!p) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    if (s) seeder_matches(s, p);
    p->seeder = s;
    return KARAM_OK;
  });
}

int karam_seeder_predict(karam_seeder* s, karam_problem* p, double* out_v) {
  if (!s || !p || !out_v) return KARAM_E_INVALID;
  return guarded(p->ctx, [&] {
    need_device(p);
    seeder_matches(s, p);
    karam_seeder* keep = p->seeder;
    p->seeder = s;
    try {
      mlp_seed(p);
    } catch (...) {
      p->seeder = keep;
      throw;
    }
    p->seeder = keep;
    const int n = p->topo.n;
    unpermute(p->i_seed.as<double>(), p->t_perm.as<int>(), p->i_out.as<double>(), p->ni, p->ld,
              n, p->ctx->stream);
    ck(cudaMemcpyAsync(out_v, p->i_out.p, (size_t)p->ni * n * sizeof(double),
                       cudaMemcpyDeviceToHost, p->ctx->stream),
       "D2H seeds");
    ck(cudaStreamSynchronize(p->ctx->stream), "seeder sync");
    return KARAM_OK;
  });
}

int karam_seeder_gemm(int32_t M, int32_t N, int32_t K, const float* A, int32_t lda,
                      int32_t transA, const float* B, int32_t ldb, int32_t transB, float* C) {
  if (!A || !B || !C || M < 1 || N < 1 || K < 1) return KARAM_E_INVALID;
  return guarded(nullptr, [&] {
    const size_t na = transA ? (size_t)K * lda : (size_t)M * lda;
    const size_t nb = transB ? (size_t)N * ldb : (size_t)K * ldb;
    DBuf dA, dB, dC;
    dA.alloc(na * sizeof(float));
    dB.alloc(nb * sizeof(float));
    dC.alloc((size_t)M * N * sizeof(float));
    ck(cudaMemcpy(dA.p, A, na * sizeof(float), cudaMemcpyHostToDevice), "H2D A");
    ck(cudaMemcpy(dB.p, B, nb * sizeof(float), cudaMemcpyHostToDevice), "H2D B");
    karam::mlp_gemm(M, N, K, dA.as<float>(), lda, transA, dB.as<float>(), ldb, transB,
                    dC.as<float>(), N, 0, nullptr);
    ck(cudaMemcpy(C, dC.p, (size_t)M * N * sizeof(float), cudaMemcpyDeviceToHost), "D2H C");
    return KARAM_OK;
  });
}

int karam_last_timing(const karam_problem* p, karam_timing* out) {
  if (!p || !out) return KARAM_E_INVALID;
  *out = p->timing;
  return KARAM_OK;
}

}  // extern "C"
