// topology.hpp -- host symbolic layer of the NR inner loop (run once per topology).
//
// Produces everything the device kernels need from a karam_netlist:
//   * the SoA device tables in tensorizeNetlist order (tensors/physics_tensors.cpp:305-493);
//   * the stamp triplets in stampSoABlock order (physics/circuitsim.h:2413-2666,
//     + addDiagonalConditioning :2857) and the CSR pattern/slot map of
//     MatrixConstructor::buildPattern / CachedCsrPattern::indexOf (math/linalg.h:82-107, 281-465);
//   * the Min-Fill ordering of FactorGraph + TreewidthAnalyzer
//     (infrastructure/factor_graph.cpp:9-162, treewidth_analyzer.cpp:14-141), computed by an
//     incremental priority-queue variant with the same (fill, id) tie-break, and its
//     translation to a permutation of the unknowns;
//   * the filled L+U pattern of symbolicFactorize (math/sparse_lu.cpp:14-128);
//   * the gather tables of the evaluation kernel and the LU program of the factor kernel,
//     all expressed in the permuted index space the device works in.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/karam.h"
#include "nr_types.h"

namespace karam {

// Term codes of the gather tables: bit 31 = negative sign, bits 24..30 = kind,
// bits 0..23 = device index.
enum JKind { JK_MOS_GDS = 0, JK_MOS_GM = 1, JK_DIO_G = 2 };
enum FKind { FK_RES = 0, FK_VS = 1, FK_IS = 2, FK_CAP = 3, FK_DIO = 4, FK_MOS = 5 };
inline int32_t term(int kind, int idx, bool neg) {
  return (neg ? int32_t(0x80000000u) : 0) | (kind << 24) | (idx & 0xFFFFFF);
}

struct Triplet {
  int row, col;     // 0-based original node indices
  int f;            // position in the filled, permuted pattern
  int kind;         // stamp source (see StampSrc)
  int idx;          // device index within its table
  bool neg;
};
enum StampSrc { SS_RES, SS_VS, SS_CAP, SS_DIO, SS_MOS_GDS, SS_MOS_GM, SS_MOS_GMB, SS_GMIN };

struct Topology {
  int n = 0;  // unknowns
  double temp_k = 300.15;

  // ---- SoA device tables (tensorised order); node ids 1-based, 0 = ground ----
  struct Mos { int d, g, s, b; double wl, w, l, kp_card, vto_card, lam; bool pmos; };
  struct Dio { int a, c; double is, n, vt; };
  struct Two { int n1, n2; double val; };
  struct Vs { int pos, neg, kind; double dc; double pulse[7]; };
  std::vector<Mos> mos;
  std::vector<Dio> dio;
  std::vector<Two> res, cap, isrc;
  std::vector<Vs> vs;
  std::vector<int> mos_order, dio_order;   // soa index -> netlist index
  std::vector<int> seed_anodes;            // netlist-order diode anodes (seedInitialGuess)

  // ---- CSR pattern (original order, transient pattern incl. gmin diagonal) ----
  std::vector<int> row_ptr, col;
  std::vector<Triplet> trip;  // stamp slots in reference order
  std::vector<int> slot_csr;  // slot -> CSR index

  // ---- ordering ----
  std::vector<uint32_t> raw_order;
  int treewidth = 0;
  std::vector<int> perm, iperm;  // perm[new] = old (0-based), iperm[old] = new

  // ---- filled pattern (permuted) ----
  std::vector<int> f_row_ptr, f_col;
  int fill_in = 0;
  std::vector<int> f_diag;  // filled position of (k, k)

  // ---- value slots: filled positions the static-pivot elimination can make
  //      non-zero (the unsymmetric stamp structure + its fill), row-major ----
  int nv = 0;
  std::vector<int> f_slot;                   // filled position -> slot (-1: always zero)
  std::vector<int> slot_row, slot_col;       // permuted (row, col) per slot

  // ---- gather tables (permuted space) ----
  std::vector<int> jt_off, jt_code;          // device terms per slot
  std::vector<double> jlin_dc;               // R + V stamps per slot
  std::vector<int> jcap_off, jcap_code;      // capacitor stamps per slot (G = 2C / h_eff)
  std::vector<int> ft_off, ft_code;          // per permuted node

  // ---- LU program: per pivot k (off, nL, nU, diagonal slot); data at off =
  //      Lrow[nL] Lslot[nL] Ucol[nU] Uslot[nU] T[nL*nU] (update target slots, row-major) ----
  std::vector<int> lu_hdr;   // 4 ints per pivot
  std::vector<int> lu_data;
  bool lu_small = false;     // every pivot has nL <= 1 and nU <= 2
  std::vector<int> lu_rec;   // pivot records (8 ints per pivot) when lu_small
  std::vector<int> lu_rec2;  // back-substitution columns (2 ints per pivot) when lu_small
  int lu_ops = 0;
  int max_d = 0;

  // ---- level-scheduled LU of the factor/solve kernel: the same static-pivot
  //      elimination on a nested-dissection order of the Min-Fill unknowns
  //      (hubs last), whose elimination tree is shallow; its own value slots
  //      ("ND slots", row-major), gathered from the Min-Fill value slots ----
  int nd_levels = 0;                 // 0: no schedule
  int nd_nv = 0;
  std::vector<int> nd_perm, nd_pos;  // ND position -> Min-Fill index, and back
  std::vector<int> nd_src;           // ND slot -> Min-Fill value slot (-1: starts at 0)
  std::vector<int> nd_diag;          // ND pivot -> ND slot of its diagonal
  // per level (CSR offsets lv_*[level .. level + 1]):
  std::vector<int> lv_piv, lv_piv_ptr;   // pivots
  std::vector<int> lv_l_ptr, l_slot, l_piv;  // L entries: l = A[slot] * reciprocal of pivot
  std::vector<int> lv_ts_ptr, lv_tl_ptr;     // update targets, short lists then long lists
  std::vector<int> t_slot, t_off;            // target slot, its pairs [t_off[t], t_off[t + 1])
  std::vector<int> pr_l, pr_u;               // pairs: L slot, U slot
  std::vector<int> lv_ys_ptr, lv_yl_ptr;     // right-hand-side rows, short then long
  std::vector<int> y_row, y_off;             // row, its pairs [y_off[r], y_off[r + 1])
  std::vector<int> yp_l, yp_k;               // pairs: L slot, pivot
  std::vector<int> bs_off, bs_u, bs_c;       // back substitution per pivot: U slots and columns
  static constexpr int kNdLong = 8;          // longer contribution lists are summed by the warp
  // The same schedule packed for shared memory (16-bit fields, two per int;
  // empty when some index does not fit 16 bits): see nd_program in
  // topology.cpp for the layout.
  std::vector<int> nd_prog;

  // ---- evaluation + stamping blocks: the stamp items (value slots 0..nv-1,
  //      nodes nv..nv+n-1) packed in row order into blocks whose devices fit
  //      one CTA's shared memory; items with more devices than that (hubs)
  //      form groups whose devices are split into chunks, one block per
  //      chunk ----
  std::vector<int> ft_a, ft_b;              // per KCL term: element terminals (permuted, -1 ground)
  std::vector<double> ft_coef;              // 1/R, source amplitude, 2C or 0
  std::vector<int> es_block;                // 4 per block: item offset, items, device offset, devices
  std::vector<int> es_item;                 // 4 per item: item id, term offset, terms, 0
  std::vector<int> es_dev;                  // global device ids (MOSFETs, then n_mos + diode)
  std::vector<int> es_jt;                   // slot device terms: sign | kind << 24 | local device
  std::vector<int> es_ft;                   // node terms: 4 per term {code, a, b, 0}; device codes
                                            // carry the local device index
  std::vector<double> es_fc;                // node term coefficients
  std::vector<int> es_hub;                  // per hub item: term index where each device
                                            // chunk starts, then the end (offset in es_item w)
  std::vector<int> es_hubc;                 // 4 per block: chunk, chunks of the group, group,
                                            // first partial row of the group (0s: not a hub block)
  int es_max_dev = 0;                       // devices per chunk (shared-memory budget)
  int n_hub_groups = 0;                     // hub groups
  int n_hub_rows = 0;                       // chunk partial rows: sum over groups of items x chunks

  // ---- junction limiting (SoA diode order) ----
  std::vector<double> dio_lim;  // 2 per diode: Vt * T/Tnom, vcrit
  std::vector<int> dio_level;   // diodes of one level share no node
  int n_dio_levels = 0;

  // ---- device tables in permuted node indices (-1 = ground) ----
  std::vector<int> mos_term;  // 4 per MOSFET: d g s b
  std::vector<int> dio_term;  // 2 per diode
  std::vector<int> res_term, cap_term, vs_term, is_term;

  int nnz() const { return (int)col.size(); }
  int nnz_filled() const { return (int)f_col.size(); }
};

// Builds the full topology; throws std::runtime_error with a message on bad input.
Topology build_topology(const karam_netlist* nl);

// Devices one evaluation + stamping CTA holds in shared memory at a time, and
// items of one evaluation + stamping block (nr_types.h).
constexpr int kEsMaxDev = KES_MAX_DEV;
constexpr int kEsMaxItems = KES_MAX_ITEMS;
constexpr int kEsMaxHubs = KES_MAX_HUBS;

// Min-Fill on an explicit factor list (exposed for tests of the ordering).
struct MinFillResult {
  std::vector<uint32_t> ordering;
  int treewidth = 0;
};
MinFillResult min_fill(const std::vector<std::vector<uint32_t>>& factors,
                       const std::vector<uint32_t>& variables);

}  // namespace karam
