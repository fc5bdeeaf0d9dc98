// spice.cpp -- SPICE netlist front-end of the C ABI (karam_spice_*).
//
// Reads the SPICE subset the batched engine solves into a karam_netlist, in
// the order of SPICEParser::parse (netlist/spice_parser.cpp:148-262): the
// first line is the title; '*' starts a comment line and ';' an inline
// comment; '+' continues the previous line; '(' ')' ',' '=' separate tokens;
// node "0" / GND / VSS / GROUND is ground and other names are numbered from 1
// in order of first appearance, case-insensitively (:78-90); values take the
// engineering suffixes of SPICEParser::parseValue (:48-76).
//
// Elements: R, C, V (DC, bare value, PULSE), I (DC, bare value), D
// (model), M (model, W, L). Directives: .MODEL (NMOS / PMOS: KP, VTO,
// LAMBDA; D: IS, N), .TEMP (Celsius), .OP, .TRAN step stop [start], .END;
// .OPTION(S), .INCLUDE, .LIB, .GLOBAL, .PARAM and .AC / .DC are skipped as in the
// reference. Anything the engine cannot solve (inductors, controlled sources,
// BJTs, JFETs, transmission lines, subcircuits, SIN sources, pulsed current
// sources) is an error naming the line, where the reference would warn and
// skip the element.
//
// The reference parser's defects are not reproduced:
//  - key=value parameters: its tokenizer turns '=' into a blank (:42-45), so
//    the "W=" / "L=" tests of parseMosfet (:494-495) never match and MOSFETs
//    keep the default 1u x 1u; here W and L are read.
//  - diode model cards: parseDiode keeps only the model name (:465-478), so
//    parsed diodes carry no Is / N; here they come from the .MODEL D card
//    (defaults 1e-14 A and 1.0; Vt 0.02585 V as TensorBlock::addDiode,
//    netlist/circuit.h:815).
//  - model lookup: cards are keyed upper-case (:649) while tensorizeNetlist
//    looks them up in the instance's spelling (tensors/physics_tensors.cpp:428);
//    here every lookup is case-insensitive.
//  - SIN: parseVoltSrc labels sine sources "SIN" (:374) where the simulator's
//    waveform is "SINE" (netlist/circuit.h:147); both spellings are recognised
//    here (and rejected, as above).
//  - title: the reference drops comment lines before it skips the title
//    (:158-166), so a title line starting with '*' takes the first element
//    with it; here the first physical line is the title, as in SPICE.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/karam.h"

struct karam_spice {
  // arrays the netlist points into
  std::vector<int32_t> vs_pos, vs_neg, vs_kind, is_pos, is_neg, r_n1, r_n2, c_n1, c_n2, d_anode,
      d_cathode, d_model, m_d, m_g, m_s, m_b, m_model, model_type;
  std::vector<double> vs_dc, vs_pulse, is_amp, r_ohm, c_farad, d_is, d_n, d_vt, m_w, m_l, model_kp,
      model_vto, model_lambda;
  std::vector<std::string> model_names;
  std::vector<const char*> model_name_ptrs;
  std::vector<std::string> node_names;  // index i - 1 -> name (upper case)
  karam_netlist nl{};
  int32_t has_op = 0, has_tran = 0;
  double tran_step = 0.0, tran_stop = 0.0, tran_start = 0.0;
};

namespace {

std::string upper(std::string s) {
  for (char& c : s) c = (char)std::toupper((unsigned char)c);
  return s;
}

struct Line {
  int num;
  std::string text;
};

// The lines after the title (the first physical line, whatever it holds),
// with comments removed and '+' continuations joined (spice_parser.cpp:95-139)
std::vector<Line> logical_lines(const char* text) {
  std::vector<Line> out;
  std::istringstream in(text);
  std::string raw;
  int num = 0;
  while (std::getline(in, raw)) {
    if (++num == 1) continue;
    const size_t semi = raw.find(';');
    if (semi != std::string::npos) raw.resize(semi);
    while (!raw.empty() && std::isspace((unsigned char)raw.back())) raw.pop_back();
    if (raw.empty() || raw[0] == '*') continue;
    if (raw[0] == '+' && !out.empty()) {
      out.back().text += " " + raw.substr(1);
      continue;
    }
    out.push_back({num, raw});
  }
  return out;
}

std::vector<std::string> tokens(const std::string& line) {
  std::string flat = line;
  for (char& c : flat)
    if (c == '(' || c == ')' || c == ',' || c == '=') c = ' ';
  std::istringstream in(flat);
  std::vector<std::string> t;
  std::string w;
  while (in >> w) t.push_back(w);
  return t;
}

// A number with an optional engineering suffix (MEG, MIL, T G K M U N P F A;
// trailing unit letters after the suffix are ignored).
double value(const std::string& s) {
  const char* b = s.c_str();
  char* e = nullptr;
  double v = std::strtod(b, &e);
  if (e == b) throw std::runtime_error("not a number: '" + s + "'");
  const std::string sfx = upper(std::string(e));
  if (sfx.empty()) return v;
  if (sfx.rfind("MEG", 0) == 0) return v * 1e6;
  if (sfx.rfind("MIL", 0) == 0) return v * 25.4e-6;
  switch (sfx[0]) {
    case 'T': return v * 1e12;
    case 'G': return v * 1e9;
    case 'K': return v * 1e3;
    case 'M': return v * 1e-3;
    case 'U': return v * 1e-6;
    case 'N': return v * 1e-9;
    case 'P': return v * 1e-12;
    case 'F': return v * 1e-15;
    case 'A': return v * 1e-18;
    default: return v;
  }
}

struct Parser {
  karam_spice& S;
  std::map<std::string, int> nodes;  // upper-case name -> index
  struct Card {
    std::string name, type;
    std::map<std::string, double> p;
  };
  std::map<std::string, Card> cards;  // upper-case name -> card
  // devices wait for the model cards, which may follow them
  struct PendingDiode {
    int a, c;
    std::string model;
    int line;
  };
  struct PendingMos {
    int d, g, s, b;
    double w, l;
    std::string model;
    int line;
  };
  int cur_line = 0;
  std::vector<PendingDiode> diodes;
  std::vector<PendingMos> mosfets;
  double temp_k = 300.15;

  int node(const std::string& name) {
    const std::string u = upper(name);
    if (u == "0" || u == "GND" || u == "VSS" || u == "GROUND") return 0;
    auto it = nodes.find(u);
    if (it != nodes.end()) return it->second;
    const int idx = (int)nodes.size() + 1;
    nodes[u] = idx;
    S.node_names.push_back(u);
    return idx;
  }

  static void need(const std::vector<std::string>& t, size_t n, const char* what) {
    if (t.size() < n) throw std::runtime_error(std::string(what) + ": too few fields");
  }

  void element(const std::vector<std::string>& t) {
    const std::string kw = upper(t[0]);
    switch (kw[0]) {
      case 'R':
        need(t, 4, "resistor");
        S.r_n1.push_back(node(t[1]));
        S.r_n2.push_back(node(t[2]));
        S.r_ohm.push_back(value(t[3]));
        return;
      case 'C':
        need(t, 4, "capacitor");
        S.c_n1.push_back(node(t[1]));
        S.c_n2.push_back(node(t[2]));
        S.c_farad.push_back(value(t[3]));
        return;
      case 'V': {
        need(t, 3, "voltage source");
        const int p = node(t[1]), q = node(t[2]);
        double dc = 0.0;
        int kind = KARAM_SRC_DC;
        double pulse[7] = {0, 0, 0, 0, 0, 0, 0};
        for (size_t i = 3; i < t.size();) {
          const std::string k = upper(t[i]);
          if (k == "DC" && i + 1 < t.size()) {
            dc = value(t[i + 1]);
            i += 2;
          } else if (k == "AC") {  // small-signal magnitude / phase: no DC effect
            i += 2;
            if (i < t.size() && (std::isdigit((unsigned char)t[i][0]) || t[i][0] == '-' || t[i][0] == '.'))
              ++i;
          } else if (k == "PULSE") {
            kind = KARAM_SRC_PULSE;
            for (int j = 0; j < 7 && i + 1 + j < t.size(); ++j) pulse[j] = value(t[i + 1 + j]);
            dc = pulse[0];  // the DC operating point sees v1 (the value at t = 0)
            i = t.size();
          } else if (k == "SIN" || k == "SINE") {
            throw std::runtime_error("SIN sources are not supported by the batched engine");
          } else {
            dc = value(t[i]);
            ++i;
          }
        }
        S.vs_pos.push_back(p);
        S.vs_neg.push_back(q);
        S.vs_dc.push_back(dc);
        S.vs_kind.push_back(kind);
        S.vs_pulse.insert(S.vs_pulse.end(), pulse, pulse + 7);
        return;
      }
      case 'I': {
        need(t, 3, "current source");
        const int p = node(t[1]), q = node(t[2]);
        double amp = 0.0;
        for (size_t i = 3; i < t.size();) {
          const std::string k = upper(t[i]);
          if (k == "DC" && i + 1 < t.size()) {
            amp = value(t[i + 1]);
            i += 2;
          } else if (k == "PULSE" || k == "SIN" || k == "SINE") {
            throw std::runtime_error("time-varying current sources are not supported by the batched engine");
          } else {
            amp = value(t[i]);
            ++i;
          }
        }
        S.is_pos.push_back(p);
        S.is_neg.push_back(q);
        S.is_amp.push_back(amp);
        return;
      }
      case 'D':
        need(t, 4, "diode");
        diodes.push_back({node(t[1]), node(t[2]), upper(t[3]), cur_line});
        return;
      case 'M': {
        need(t, 6, "MOSFET");
        PendingMos m{node(t[1]), node(t[2]), node(t[3]), node(t[4]), 1e-6, 1e-6, upper(t[5]), cur_line};
        for (size_t i = 6; i + 1 < t.size(); i += 2) {  // KEY VALUE pairs (KEY=VALUE)
          const std::string k = upper(t[i]);
          if (k == "W")
            m.w = value(t[i + 1]);
          else if (k == "L")
            m.l = value(t[i + 1]);
        }
        mosfets.push_back(m);
        return;
      }
      default:
        throw std::runtime_error("element '" + t[0] + "' is not supported by the batched engine");
    }
  }

  void directive(const std::vector<std::string>& t) {
    const std::string kw = upper(t[0]);
    if (kw == ".MODEL") {
      need(t, 3, ".MODEL");
      Card c{t[1], upper(t[2]), {}};
      for (size_t i = 3; i + 1 < t.size(); i += 2) c.p[upper(t[i])] = value(t[i + 1]);
      cards[upper(t[1])] = c;
    } else if (kw == ".TEMP") {
      need(t, 2, ".TEMP");
      temp_k = 273.15 + value(t[1]);
    } else if (kw == ".OP") {
      S.has_op = 1;
    } else if (kw == ".TRAN") {
      S.has_tran = 1;
      if (t.size() >= 3) {
        S.tran_step = value(t[1]);
        S.tran_stop = value(t[2]);
        if (t.size() >= 4) S.tran_start = value(t[3]);
      }
    } else if (kw == ".SUBCKT" || kw == ".ENDS") {
      throw std::runtime_error("subcircuits are not supported by the batched engine");
    }
    // .OPTION(S), .INCLUDE, .LIB, .GLOBAL, .PARAM, .AC, .DC: skipped
  }

  // model cards in name order (the reference merges its std::map of cards,
  // spice_parser.cpp:251-255); only the kinds the engine evaluates
  void finish() {
    std::map<std::string, int> index;
    for (const auto& kv : cards) {
      const Card& c = kv.second;
      int type;
      if (c.type == "NMOS")
        type = KARAM_MODEL_NMOS;
      else if (c.type == "PMOS")
        type = KARAM_MODEL_PMOS;
      else if (c.type == "D")
        type = KARAM_MODEL_DIODE;
      else
        continue;
      const double nan = std::numeric_limits<double>::quiet_NaN();
      auto get = [&](const char* k) {
        auto it = c.p.find(k);
        return it == c.p.end() ? nan : it->second;
      };
      index[kv.first] = (int)S.model_type.size();
      S.model_names.push_back(c.name);
      S.model_type.push_back(type);
      S.model_kp.push_back(get("KP"));
      S.model_vto.push_back(get("VTO"));
      S.model_lambda.push_back(get("LAMBDA"));
    }
    auto undefined = [](int line, const char* what, const std::string& name) {
      return std::runtime_error("line " + std::to_string(line) + ": " + what + " model '" + name +
                                "' is not defined");
    };
    for (const PendingDiode& d : diodes) {
      auto itd = index.find(d.model);
      if (itd == index.end() || S.model_type[itd->second] != KARAM_MODEL_DIODE)
        throw undefined(d.line, "diode", d.model);
      const int mi = itd->second;
      const Card& c = cards.at(d.model);
      auto it_is = c.p.find("IS"), it_n = c.p.find("N");
      S.d_anode.push_back(d.a);
      S.d_cathode.push_back(d.c);
      S.d_is.push_back(it_is == c.p.end() ? 1e-14 : it_is->second);
      S.d_n.push_back(it_n == c.p.end() ? 1.0 : it_n->second);
      S.d_vt.push_back(0.02585);
      S.d_model.push_back(mi);
    }
    for (const PendingMos& m : mosfets) {
      auto it = index.find(m.model);
      if (it == index.end() || S.model_type[it->second] == KARAM_MODEL_DIODE)
        throw undefined(m.line, "MOSFET", m.model);
      S.m_d.push_back(m.d);
      S.m_g.push_back(m.g);
      S.m_s.push_back(m.s);
      S.m_b.push_back(m.b);
      S.m_w.push_back(m.w);
      S.m_l.push_back(m.l);
      S.m_model.push_back(it->second);
    }
    for (const std::string& n : S.model_names) S.model_name_ptrs.push_back(n.c_str());
    karam_netlist& nl = S.nl;
    nl.n_nodes = (int)nodes.size();
    nl.temp_k = temp_k;
    auto ip = [](const std::vector<int32_t>& v) { return v.empty() ? nullptr : v.data(); };
    auto dp = [](const std::vector<double>& v) { return v.empty() ? nullptr : v.data(); };
    nl.n_vsrc = (int)S.vs_pos.size();
    nl.vs_pos = ip(S.vs_pos);
    nl.vs_neg = ip(S.vs_neg);
    nl.vs_dc = dp(S.vs_dc);
    nl.vs_kind = ip(S.vs_kind);
    nl.vs_pulse = dp(S.vs_pulse);
    nl.n_isrc = (int)S.is_pos.size();
    nl.is_pos = ip(S.is_pos);
    nl.is_neg = ip(S.is_neg);
    nl.is_amp = dp(S.is_amp);
    nl.n_res = (int)S.r_n1.size();
    nl.r_n1 = ip(S.r_n1);
    nl.r_n2 = ip(S.r_n2);
    nl.r_ohm = dp(S.r_ohm);
    nl.n_cap = (int)S.c_n1.size();
    nl.c_n1 = ip(S.c_n1);
    nl.c_n2 = ip(S.c_n2);
    nl.c_farad = dp(S.c_farad);
    nl.n_dio = (int)S.d_anode.size();
    nl.d_anode = ip(S.d_anode);
    nl.d_cathode = ip(S.d_cathode);
    nl.d_is = dp(S.d_is);
    nl.d_n = dp(S.d_n);
    nl.d_vt = dp(S.d_vt);
    nl.d_model = ip(S.d_model);
    nl.n_mos = (int)S.m_d.size();
    nl.m_d = ip(S.m_d);
    nl.m_g = ip(S.m_g);
    nl.m_s = ip(S.m_s);
    nl.m_b = ip(S.m_b);
    nl.m_w = dp(S.m_w);
    nl.m_l = dp(S.m_l);
    nl.m_model = ip(S.m_model);
    nl.n_models = (int)S.model_type.size();
    nl.model_name = S.model_name_ptrs.empty() ? nullptr : S.model_name_ptrs.data();
    nl.model_type = ip(S.model_type);
    nl.model_kp = dp(S.model_kp);
    nl.model_vto = dp(S.model_vto);
    nl.model_lambda = dp(S.model_lambda);
  }
};

void put_error(char* err, int32_t len, const std::string& msg) {
  if (!err || len <= 0) return;
  const size_t n = std::min<size_t>(msg.size(), (size_t)len - 1);
  std::memcpy(err, msg.data(), n);
  err[n] = 0;
}

}  // namespace

extern "C" {

int karam_spice_parse(const char* text, karam_spice** out, char* err, int32_t err_len) {
  if (!text || !out) return KARAM_E_INVALID;
  *out = nullptr;
  auto* S = new karam_spice();
  Parser P{*S};
  int line_num = 0;
  try {
    if (!*text) throw std::runtime_error("empty netlist");
    const std::vector<Line> lines = logical_lines(text);
    for (size_t k = 0; k < lines.size(); ++k) {
      line_num = P.cur_line = lines[k].num;
      const std::vector<std::string> t = tokens(lines[k].text);
      if (t.empty()) continue;
      if (t[0][0] == '.') {
        if (upper(t[0]) == ".END") break;
        P.directive(t);
      } else {
        P.element(t);
      }
    }
    line_num = 0;
    P.finish();
  } catch (const std::exception& e) {
    put_error(err, err_len,
              line_num ? "line " + std::to_string(line_num) + ": " + e.what() : std::string(e.what()));
    delete S;
    return KARAM_E_INVALID;
  }
  *out = S;
  return KARAM_OK;
}

const karam_netlist* karam_spice_netlist(const karam_spice* s) { return s ? &s->nl : nullptr; }

int32_t karam_spice_node(const karam_spice* s, const char* name) {
  if (!s || !name) return -1;
  std::string u(name);
  for (char& c : u) c = (char)std::toupper((unsigned char)c);
  if (u == "0" || u == "GND" || u == "VSS" || u == "GROUND") return 0;
  for (size_t i = 0; i < s->node_names.size(); ++i)
    if (s->node_names[i] == u) return (int32_t)i + 1;
  return -1;
}

int karam_spice_analysis(const karam_spice* s, int32_t* has_op, int32_t* has_tran, double* tran_step,
                         double* tran_stop, double* tran_start) {
  if (!s) return KARAM_E_INVALID;
  if (has_op) *has_op = s->has_op;
  if (has_tran) *has_tran = s->has_tran;
  if (tran_step) *tran_step = s->tran_step;
  if (tran_stop) *tran_stop = s->tran_stop;
  if (tran_start) *tran_start = s->tran_start;
  return KARAM_OK;
}

void karam_spice_free(karam_spice* s) { delete s; }

}  // extern "C"
