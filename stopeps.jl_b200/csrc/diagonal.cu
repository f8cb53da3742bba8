// Diagonal boundary-MPS contraction on the Z2 engine (BoundaryMPSDiagonal):
// restates src/contraction/diagonal_mps.jl, the Born sampling of
// src/sampling/diagonal_born.jl and the energy of
// src/measurement/diagonal_energy.jl.
//
// The lattice is swept by anti-diagonal layers t = x + y (0-based sites; the
// reference's t - 2, so the parity of t agrees).  A layer is absorbed as one
// raw block per site: the frontier tensors of the site's input edges
// contracted with its ket, then its bra.  The blocks are put in an exact
// canonical form and only the bond a site opens between its two output
// edges is truncated (the bonds between blocks already meet the budget).
// Strips of one or two layers between cached boundaries carry the sampling
// conditionals and the energy terms.  Networks are built from labelled
// tensors that contract every label they share; every contraction is the
// engine's table-addressed ein, every factorization its QR/LQ/SVD.
#include "pipeline.h"
#include <algorithm>
#include <cfloat>

namespace sps {
namespace {

const int VAX[4] = {0, 1, 4, 5};   // w, n, e, s legs of a site tensor (w, n, p, a, e, s)
const int PHYS = -21, AUX = -22;   // physical and auxiliary legs shared by ket and bra
const int LBL = 1 << 24, RBL = LBL + 1, R2L = LBL + 2;   // raw-block chain ends
const int BOND = 1 << 20;          // strip labels of boundary bonds

// _DiagonalTensor (diagonal_mps.jl:14-20): a tensor with one label per leg,
// or a plain number
struct LT {
  Tensor t;
  std::vector<int> lab;
  bool number = false;
  bool unit = false;   // every leg one-dimensional and even, value 1
  double s = 1.0;
};

LT number(double v) {
  LT a;
  a.number = true;
  a.s = v;
  return a;
}

int index_of(const std::vector<int>& v, int x) {
  auto it = std::find(v.begin(), v.end(), x);
  return it == v.end() ? -1 : (int)(it - v.begin());
}

char letter(int i) {
  if (i < 26) return (char)('a' + i);
  if (i < 52) return (char)('A' + i - 26);
  throw Error(SPS_ERR_ARGUMENT, "diagonal network: too many legs");
}

// the engine, the lattice's edge labels (_diagonal_ports,
// diagonal_mps.jl:91-97) and a unit vector for open-boundary legs
struct Net {
  Engine& E;
  int Lx, Ly;
  Par triv;
  Tensor u1;
  Net(Engine& e, int lx, int ly) : E(e), Lx(lx), Ly(ly), triv(make_par(1, 0)) { u1 = unit_tensor(E, {triv}); }
  int hedge(int x, int y) const { return 1 + x + y * (Lx + 1); }             // (x-1,y)-(x,y), x = 0..Lx
  int vedge(int x, int y) const { return 1 + (Lx + 1) * Ly + x + y * Lx; }   // (x,y-1)-(x,y), y = 0..Ly
  std::array<int, 4> ports(int x, int y) const { return {hedge(x, y), vedge(x, y), hedge(x + 1, y), vedge(x, y + 1)}; }
  std::array<bool, 4> inside(int x, int y) const { return {x > 0, y > 0, x < Lx - 1, y < Ly - 1}; }
  LT unit(int label) const {
    LT a;
    a.t = u1;
    a.lab = {label};
    a.unit = true;
    return a;
  }
};

// A with `count` trivial legs added in front or at the back (a view)
Tensor with_trivial(const Tensor& A, int count, bool front, const Par& triv) {
  Tensor t = A;
  const int64_t size = std::max<int64_t>(A.size(), 1);
  for (int i = 0; i < count; ++i) {
    if (front) {
      t.legs.insert(t.legs.begin(), triv);
      t.dims.insert(t.dims.begin(), 1);
      t.strides.insert(t.strides.begin(), size);
    } else {
      t.legs.push_back(triv);
      t.dims.push_back(1);
      t.strides.push_back(1);
    }
  }
  return t;
}

// _diagonal_join (diagonal_mps.jl:21-28): contract the shared labels; the
// result keeps a's free labels, then b's
LT join(Net& n, const LT& a, const LT& b) {
  Engine& E = n.E;
  if (a.number || b.number) {
    if (a.number && b.number) return number(a.s * b.s);
    const LT& t = a.number ? b : a;
    const double f = a.number ? a.s : b.s;
    if (f == 1.0) return t;
    LT r = t;
    r.t = clone(E, t.t);
    scale_inplace(E, r.t, f);
    r.unit = false;
    return r;
  }
  std::vector<int> common, fa, fb;
  for (int k : a.lab) (index_of(b.lab, k) >= 0 ? common : fa).push_back(k);
  for (int k : b.lab)
    if (index_of(a.lab, k) < 0) fb.push_back(k);
  if (fa.empty() && fb.empty()) {   // a closed network
    std::vector<int> order;
    for (int i = 0; i < (int)b.lab.size(); ++i) {
      const int j = index_of(a.lab, b.lab[i]);
      if (a.t.dims[j] != b.t.dims[i] || *a.t.legs[j] != *b.t.legs[i])
        throw Error(SPS_ERR_ARGUMENT, "diagonal network: leg mismatch in a closed contraction");
      order.push_back(j);
    }
    return number(dot(E, perm_view(a.t, order), b.t));
  }
  if (common.empty()) {
    // outer products only meet unit vectors here: add their trivial legs
    LT r;
    r.lab = a.lab;
    r.lab.insert(r.lab.end(), b.lab.begin(), b.lab.end());
    if (b.unit) {
      r.t = with_trivial(a.t, (int)b.lab.size(), false, n.triv);
      r.unit = a.unit;
    } else if (a.unit) {
      r.t = with_trivial(b.t, (int)a.lab.size(), true, n.triv);
    } else {
      throw Error(SPS_ERR_ARGUMENT, "diagonal network: disconnected tensors");
    }
    return r;
  }
  std::vector<int> all = a.lab;
  all.insert(all.end(), fb.begin(), fb.end());
  std::string spec;
  for (int k : a.lab) spec += letter(index_of(all, k));
  spec += ',';
  for (int k : b.lab) spec += letter(index_of(all, k));
  spec += "->";
  LT r;
  for (int k : fa) {
    spec += letter(index_of(all, k));
    r.lab.push_back(k);
  }
  for (int k : fb) {
    spec += letter(index_of(all, k));
    r.lab.push_back(k);
  }
  r.t = ein(E, spec, a.t, b.t);
  return r;
}

LT labelled(const Tensor& t, std::vector<int> lab) {
  LT a;
  a.t = t;
  a.lab = std::move(lab);
  return a;
}

// _diagonal_reorder (a view)
Tensor reordered(const LT& a, const std::vector<int>& labels) {
  if (labels.size() != a.lab.size()) throw Error(SPS_ERR_ARGUMENT, "diagonal tensor labels");
  std::vector<int> order;
  for (int k : labels) {
    const int i = index_of(a.lab, k);
    if (i < 0) throw Error(SPS_ERR_ARGUMENT, "diagonal tensor labels");
    order.push_back(i);
  }
  return perm_view(a.t, order);
}

// _diagonal_apply (diagonal_mps.jl:58-88): contract the two input ports of
// `msg` with the ket A, then the bra B; the other two virtual legs leave as
// fused (ket, bra) ports, appended in w, n, e, s order.  `phys` (two labels)
// keeps the physical legs open.
LT apply(Net& n, LT msg, const Tensor& A, const Tensor& B, const std::array<int, 4>& ports,
         const std::vector<int>& inputs, const int* phys = nullptr) {
  if (inputs.size() != 2) throw Error(SPS_ERR_ARGUMENT, "a diagonal vertex has two input ports");
  int rk[6] = {-1, -2, PHYS, AUX, -5, -6}, rb[6] = {-11, -12, PHYS, AUX, -15, -16};
  if (phys) {
    rk[2] = phys[0];
    rb[2] = phys[1];
  }
  for (int port : inputs) {
    const int j = (int)(std::find(ports.begin(), ports.end(), port) - ports.begin());
    const int axis = VAX[j];
    const int pos = index_of(msg.lab, port);
    if (pos < 0 || *msg.t.legs[pos] != *fused_par({A.legs[axis], B.legs[axis]}))
      throw Error(SPS_ERR_ARGUMENT, "diagonal network: input port does not match the site's legs");
    msg.t = split(n.E, msg.t, pos, {A.legs[axis], B.legs[axis]});
    msg.lab.erase(msg.lab.begin() + pos);
    msg.lab.insert(msg.lab.begin() + pos, {rk[axis], rb[axis]});
    msg.unit = false;
  }
  msg = join(n, msg, labelled(A, std::vector<int>(rk, rk + 6)));
  msg = join(n, msg, labelled(B, std::vector<int>(rb, rb + 6)));
  for (int j = 0; j < 4; ++j) {
    const int port = ports[j];
    if (std::find(inputs.begin(), inputs.end(), port) != inputs.end()) continue;
    const int axis = VAX[j];
    std::vector<int> others, order;
    for (int i = 0; i < (int)msg.lab.size(); ++i)
      if (msg.lab[i] != rk[axis] && msg.lab[i] != rb[axis]) {
        others.push_back(msg.lab[i]);
        order.push_back(i);
      }
    order.push_back(index_of(msg.lab, rk[axis]));
    order.push_back(index_of(msg.lab, rb[axis]));
    msg.t = fuse(n.E, perm_view(msg.t, order), (int)others.size(), 2);
    others.push_back(port);
    msg.lab = others;
  }
  return msg;
}

// sites of layer t by increasing x - y (increasing x)
std::vector<std::array<int, 2>> layer_sites(int Lx, int Ly, int t) {
  std::vector<std::array<int, 2>> out;
  for (int x = std::max(0, t - Ly + 1); x <= std::min(Lx - 1, t); ++x) out.push_back({x, t - x});
  return out;
}

struct Layout {   // _diagonal_layer_layout (diagonal_mps.jl:158-176)
  std::vector<std::array<int, 2>> sites;
  std::vector<std::vector<int>> inputs, outputs, ranges;
  std::vector<int> edges;
};

Layout layer_layout(const Net& n, const DiagEnv& inp, int t, bool reverse) {
  Layout L;
  L.sites = layer_sites(n.Lx, n.Ly, t);
  const int ia[2] = {reverse ? 3 : 0, reverse ? 2 : 1};
  const int oa[2] = {reverse ? 0 : 3, reverse ? 1 : 2};
  for (auto& s : L.sites) {
    auto ports = n.ports(s[0], s[1]);
    auto inside = n.inside(s[0], s[1]);
    std::vector<int> incoming, out, idx, range;
    for (int k : ia)
      if (inside[k]) incoming.push_back(ports[k]);
    const int p = incoming.empty() ? 0 : index_of(inp.edges, incoming[0]);
    for (int i = 0; i < (int)incoming.size(); ++i) {
      if (p < 0 || p + i >= (int)inp.edges.size() || inp.edges[p + i] != incoming[i])
        throw Error(SPS_ERR_ARGUMENT, "nonadjacent diagonal frontier inputs");
      idx.push_back(p + i);
    }
    for (int k : oa)
      if (inside[k]) out.push_back(ports[k]);
    for (int i = 0; i < (int)out.size(); ++i) range.push_back((int)L.edges.size() + i);
    L.inputs.push_back(idx);
    L.outputs.push_back(out);
    L.ranges.push_back(range);
    L.edges.insert(L.edges.end(), out.begin(), out.end());
  }
  return L;
}

// _diagonal_raw_block (diagonal_mps.jl:179-209): legs (left, outputs..., right)
Tensor raw_block(Net& n, const DiagEnv& inp, const Tensor& A, int x, int y, const std::vector<int>& idx,
                 const std::vector<int>& outputs, bool reverse) {
  auto ports = n.ports(x, y);
  auto inside = n.inside(x, y);
  const int ia[2] = {reverse ? 3 : 0, reverse ? 2 : 1};
  const int oa[2] = {reverse ? 0 : 3, reverse ? 1 : 2};
  std::vector<int> inputs;
  for (int k : ia)
    if (inside[k]) inputs.push_back(ports[k]);
  LT phi;
  if (inputs.empty()) {
    if (!inp.t.empty()) throw Error(SPS_ERR_ARGUMENT, "disconnected diagonal initialization");
    phi = labelled(unit_tensor(n.E, {n.triv, n.triv}), {LBL, RBL});
    phi.unit = true;
  } else if (inputs.size() == 1) {
    phi = labelled(inp.t[idx[0]], {LBL, inputs[0], RBL});
  } else {
    phi = join(n, labelled(inp.t[idx[0]], {LBL, inputs[0], R2L}), labelled(inp.t[idx[1]], {R2L, inputs[1], RBL}));
  }
  for (int k : ia)
    if (!inside[k]) phi = join(n, phi, n.unit(ports[k]));
  LT theta = apply(n, phi, A, A, ports, {ports[ia[0]], ports[ia[1]]});
  for (int k : oa)
    if (!inside[k]) theta = join(n, theta, n.unit(ports[k]));
  std::vector<int> order{LBL};
  order.insert(order.end(), outputs.begin(), outputs.end());
  order.push_back(RBL);
  return contiguous(n.E, reordered(theta, order));
}

// _diagonal_normalized: A / |A| in place (A owns its buffer), log |A|
double normalize(Engine& E, Tensor& A) {
  const double s = norm(E, A);
  if (!std::isfinite(s)) throw Error(SPS_ERR_NUMERIC, "nonfinite diagonal boundary norm");
  if (s == 0) return -INFINITY;
  scale_inplace(E, A, 1.0 / s);
  return std::log(s);
}

// c = R (k, r) times the first leg of X
Tensor times_first(Engine& E, const Tensor& R, const Tensor& X) {
  std::string rest;
  for (int i = 1; i < X.rank(); ++i) rest += letter(2 + i);
  return ein(E, "ab,b" + rest + "->a" + rest, R, X);
}

// c = the last leg of X times L (l, k)
Tensor times_last(Engine& E, const Tensor& X, const Tensor& L) {
  std::string rest;
  for (int i = 0; i + 1 < X.rank(); ++i) rest += letter(2 + i);
  return ein(E, rest + "a,ab->" + rest + "b", X, L);
}

// _diagonal_block_center_step! (diagonal_mps.jl:219-237)
double block_center_step(Engine& E, std::vector<Tensor>& blocks, int j, bool right) {
  const Tensor& A = blocks[j];
  const int rank = A.rank();
  std::vector<int> head, tail;
  if (right) {
    for (int i = 0; i + 1 < rank; ++i) head.push_back(i);
    QRres f = qr(E, A, head, {rank - 1});
    blocks[j] = f.Q;
    Tensor R = contiguous(E, f.R);
    const double s = normalize(E, R);
    blocks[j + 1] = times_first(E, R, blocks[j + 1]);
    return s;
  }
  for (int i = 1; i < rank; ++i) tail.push_back(i);
  LQres f = lq(E, A, {0}, tail);
  blocks[j] = f.Q;
  Tensor L = contiguous(E, f.L);
  const double s = normalize(E, L);
  blocks[j - 1] = times_last(E, blocks[j - 1], L);
  return s;
}

struct Compressed {
  std::vector<Tensor> tensors;
  double log_scale = 0, max_trunc = 0;
};

// _diagonal_compress_blocks! (diagonal_mps.jl:240-271)
Compressed compress_blocks(Engine& E, std::vector<Tensor>& blocks, const Layout& L, const BMPS& m, bool right,
                           bool reverse, Entropy* ent, int Lx) {
  const int n = (int)blocks.size();
  Compressed c;
  if (right) {
    for (int j = n - 1; j >= 1; --j) c.log_scale += block_center_step(E, blocks, j, false);
  } else {
    for (int j = 0; j < n - 1; ++j) c.log_scale += block_center_step(E, blocks, j, true);
  }
  Trunc tr;
  tr.chi = m.chi;
  tr.space[0] = m.space[0];
  tr.space[1] = m.space[1];
  c.tensors.resize(L.edges.size());
  for (int step = 0; step < n; ++step) {
    const int j = right ? step : n - 1 - step;
    const auto& cut = L.ranges[j];
    if (cut.empty()) throw Error(SPS_ERR_ARGUMENT, "diagonal block without outputs");
    if (cut.size() == 2) {
      SVDres f = svd(E, blocks[j], {0, 1}, {2, 3}, tr, ent != nullptr);
      if (ent) {
        const int site = L.sites[j][0] + L.sites[j][1] * Lx;
        ent->maximum = std::max(ent->maximum, f.entropy);
        if (ent->profile) (reverse ? ent->southeast : ent->northwest)[site] = f.entropy;
      }
      c.max_trunc = std::max(c.max_trunc, f.norm == 0 ? 0.0 : (f.err / f.norm) * (f.err / f.norm));
      std::vector<double> sv(f.S[0]);
      sv.insert(sv.end(), f.S[1].begin(), f.S[1].end());
      if (right) {
        c.tensors[cut[0]] = f.U;
        blocks[j] = scale_leg(E, f.V, 0, sv);
      } else {
        c.tensors[cut[1]] = f.V;
        blocks[j] = scale_leg(E, f.U, 2, sv);
      }
    }
    if (j == (right ? n - 1 : 0)) {
      blocks[j] = contiguous(E, blocks[j]);
      c.log_scale += normalize(E, blocks[j]);
    } else {
      c.log_scale += block_center_step(E, blocks, j, right);
    }
    c.tensors[right ? cut.back() : cut.front()] = blocks[j];
  }
  return c;
}

// _diagonal_absorb_layer! (diagonal_mps.jl:272-297); site(x, y) gives the
// tensor absorbed at a site
template <class Site>
void absorb_layer_variational(Net& n, DiagEnv& env, Site site, int t, const BMPS& m, bool reverse, Entropy* ent);

template <class Site>
void absorb_layer(Net& n, DiagEnv& env, Site site, int t, const BMPS& m, bool reverse, Entropy* ent) {
  if (m.variational) return absorb_layer_variational(n, env, site, t, m, reverse, ent);
  if (m.chi < 1) throw Error(SPS_ERR_ARGUMENT, "chi must be positive");
  Layout L = layer_layout(n, env, t, reverse);
  std::vector<Tensor> blocks;
  double scale = env.log_scale;
  for (size_t j = 0; j < L.sites.size(); ++j) {
    const int x = L.sites[j][0], y = L.sites[j][1];
    Tensor A = raw_block(n, env, site(x, y), x, y, L.inputs[j], L.outputs[j], reverse);
    scale += normalize(n.E, A);
    blocks.push_back(A);
  }
  if (L.edges.empty()) {
    // the last corner: two unit boundary bonds
    if (blocks.size() != 1 || blocks[0].size() != 1) throw Error(SPS_ERR_ARGUMENT, "diagonal corner is not closed");
    env.t.clear();
    env.scalar = sum_all(n.E, blocks[0]);
  } else {
    const bool right = blocks.size() < 2 ? !reverse : ((t % 2 == 0) != reverse);
    Compressed c = compress_blocks(n.E, blocks, L, m, right, reverse, ent, n.Lx);
    env.t = c.tensors;
    env.center = right ? (int)c.tensors.size() - 1 : 0;
    env.max_trunc = std::max(env.max_trunc, c.max_trunc);
    scale += c.log_scale;
  }
  env.edges = L.edges;
  env.log_scale = scale;
}

// ---------------------------------------------------------------------------
// BoundaryMPSDiagonalVariational (src/contraction/diagonal_variational.jl): a
// layer absorbed by a two-site variational fit of the candidate frontier MPS
// to the chain of raw site blocks, normalised to unit norm.  Cross-block
// projections take the full two-site SVD (the reference's factored SVD keeps
// the same space or falls back to it); the target-block cache only saves work.
// ---------------------------------------------------------------------------

const int TB = 1 << 22, CB = 1 << 23;   // target and candidate bond labels

struct VFail : Error {   // _VariationalNumericalError
  std::string reason;
  explicit VFail(const std::string& r) : Error(SPS_ERR_NUMERIC, "variational boundary: " + r), reason(r) {}
};

struct VMsg {   // _VariationalMessage
  LT m;
  double ls = 0;
};

VMsg vmsg(Net& n, LT t, double ls = 0.0) {
  double s;
  if (t.number) {
    s = std::fabs(t.s);
  } else {
    t.t = contiguous(n.E, t.t);
    s = norm(n.E, t.t);
  }
  if (!std::isfinite(s)) throw VFail("nonfinite_overlap");
  if (s == 0) return {t, -INFINITY};
  if (t.number) {
    t.s /= s;
  } else {
    t.t = clone(n.E, t.t);
    scale_inplace(n.E, t.t, 1.0 / s);
    t.unit = false;
  }
  return {t, ls + std::log(s)};
}

// _diagonal_coordinate (diagonal_variational.jl:52-60): twice the transverse
// coordinate x - y of an edge's midpoint
int coordinate(const Net& n, int e) {
  const int nh = (n.Lx + 1) * n.Ly;
  if (e <= nh) {
    const int x = (e - 1) % (n.Lx + 1), y = (e - 1) / (n.Lx + 1);
    return 2 * x - 1 - 2 * y;
  }
  const int r = e - 1 - nh, x = r % n.Lx, y = r / n.Lx;
  return 2 * x - 2 * y + 1;
}

// _variational_identity of a single-layer leg p, on its fused (ket, bra) leg
Tensor identity_leg(Engine& E, const Par& p) {
  const int d = (int)p->size();
  std::vector<double> v((size_t)d * d, 0.0);
  for (int k = 0; k < d; ++k) v[(size_t)k * d + k] = 1.0 / std::sqrt((double)d);
  return E.upload({fused_par({p, p})}, v.data());
}

// A without its one-dimensional leg `axis` (a view)
Tensor drop_trivial(const Tensor& A, int axis) {
  if (A.dims[axis] != 1) throw Error(SPS_ERR_ARGUMENT, "diagonal variational: leg is not trivial");
  Tensor t = A;
  t.legs.erase(t.legs.begin() + axis);
  t.dims.erase(t.dims.begin() + axis);
  t.strides.erase(t.strides.begin() + axis);
  return t;
}

struct VTarget {   // _DiagonalLayerTarget (diagonal_variational.jl:96-217)
  Net& n;
  const DiagEnv& input;
  int t;
  bool reverse;
  Layout L;
  std::vector<int> owner;
  std::vector<Par> physical;
  std::vector<Par> single;     // the single-layer leg of each output edge
  std::vector<std::array<Par, 4>> legs4;   // each site's virtual legs w, n, e, s
  std::vector<Tensor> blocks;
  double log_scale = 0, weight = 1;
};

double chain_lognorm(Engine& E, const std::vector<Tensor>& blocks) {   // _variational_chain_lognorm
  Tensor carry;
  bool have = false;
  double total = 0;
  for (const Tensor& B : blocks) {
    Tensor A = have ? times_first(E, carry, B) : B;
    std::vector<int> head;
    for (int i = 0; i + 1 < A.rank(); ++i) head.push_back(i);
    QRres f = qr(E, A, head, {A.rank() - 1});
    Tensor R = contiguous(E, f.R);
    const double s = norm(E, R);
    if (!std::isfinite(s)) throw VFail("nonfinite_norm");
    if (s == 0) return -INFINITY;
    total += std::log(s);
    R = clone(E, R);
    scale_inplace(E, R, 1.0 / s);
    carry = R;
    have = true;
  }
  return total;
}

template <class Site>
VTarget make_target(Net& n, const DiagEnv& inp, Site site, int t, bool reverse) {
  VTarget g{n, inp, t, reverse, layer_layout(n, inp, t, reverse)};
  g.log_scale = inp.log_scale;
  std::vector<double> norms;
  for (size_t j = 0; j < g.L.sites.size(); ++j) {
    const int x = g.L.sites[j][0], y = g.L.sites[j][1];
    const Tensor& A = site(x, y);
    auto ports = n.ports(x, y);
    g.legs4.push_back({A.legs[0], A.legs[1], A.legs[4], A.legs[5]});
    for (int port : g.L.outputs[j]) {
      const int axis = VAX[std::find(ports.begin(), ports.end(), port) - ports.begin()];
      g.owner.push_back((int)j);
      g.physical.push_back(fused_par({A.legs[axis], A.legs[axis]}));
      g.single.push_back(A.legs[axis]);
    }
    Tensor B = raw_block(n, inp, A, x, y, g.L.inputs[j], g.L.outputs[j], reverse);
    const double s = norm(n.E, B);
    if (!std::isfinite(s)) throw Error(SPS_ERR_NUMERIC, "nonfinite variational target block");
    if (s != 0) scale_inplace(n.E, B, 1.0 / s);
    norms.push_back(s);
    g.blocks.push_back(B);
  }
  bool zero = false;
  double sumlog = 0;
  for (double s : norms) {
    zero |= s == 0;
    if (s != 0) sumlog += std::log(s);
  }
  if (zero) {
    g.log_scale = -INFINITY;
  } else if (!g.L.edges.empty()) {
    const double ln = chain_lognorm(n.E, g.blocks);
    g.log_scale += sumlog + ln;
    g.weight = std::isfinite(ln) ? std::exp(-ln / (double)g.blocks.size()) : 1.0;
    for (Tensor& B : g.blocks) scale_inplace(n.E, B, g.weight);
  } else {
    g.log_scale += sumlog;
  }
  return g;
}

LT labelled_block(const VTarget& g, int j) {
  std::vector<int> lab{TB + j};
  lab.insert(lab.end(), g.L.outputs[j].begin(), g.L.outputs[j].end());
  lab.push_back(TB + j + 1);
  return labelled(g.blocks[j], lab);
}

VMsg vedge(VTarget& g, int ncand, bool left) {   // _variational_edge
  return vmsg(g.n, join(g.n, g.n.unit(TB + (left ? 0 : (int)g.L.sites.size())), g.n.unit(CB + (left ? 0 : ncand))));
}

VMsg vstep(VTarget& g, const VMsg& m, int i, const Tensor& A, bool left) {   // _variational_step
  const int j = g.owner[i];
  const auto& rng = g.L.ranges[j];
  LT E = m.m;
  if (i == (left ? rng.front() : rng.back())) E = join(g.n, E, labelled_block(g, j));
  E = join(g.n, E, labelled(A, {CB + i, g.L.edges[i], CB + i + 1}));
  return vmsg(g.n, E, m.ls);
}

std::vector<VMsg> vmessages(VTarget& g, const DiagEnv& C, bool left) {
  const int nc = (int)C.t.size();
  std::vector<VMsg> out(nc + 1);
  if (left) {
    out[0] = vedge(g, nc, true);
    for (int i = 0; i < nc; ++i) out[i + 1] = vstep(g, out[i], i, C.t[i], true);
  } else {
    out[nc] = vedge(g, nc, false);
    for (int i = nc - 1; i >= 0; --i) out[i] = vstep(g, out[i + 1], i, C.t[i], false);
  }
  return out;
}

// _variational_pair: the two-site projection (cb_i, e_i, e_i+1, cb_i+2)
Tensor vpair(VTarget& g, int i, const VMsg& L, const VMsg& R) {
  LT E = L.m;
  std::vector<int> js{g.owner[i], g.owner[i + 1]};
  if (js[0] == js[1]) js.pop_back();
  for (int j : js) {
    const auto& rng = g.L.ranges[j];
    if (rng.front() >= i && rng.back() <= i + 1) E = join(g.n, E, labelled_block(g, j));
  }
  E = join(g.n, E, R.m);
  Tensor M = clone(g.n.E, contiguous(g.n.E, reordered(E, {CB + i, g.L.edges[i], g.L.edges[i + 1], CB + i + 2})));
  scale_inplace(g.n.E, M, std::exp(L.ls + R.ls));
  return M;
}

void vmove_center(Engine& E, DiagEnv& C, int target) {   // _diagonal_center!
  while (C.center < target) {
    const int i = C.center;
    QRres f = qr(E, C.t[i], {0, 1}, {2});
    C.t[i] = f.Q;
    C.t[i + 1] = ein(E, "lk,kpr->lpr", f.R, C.t[i + 1]);
    C.center++;
  }
  while (C.center > target) {
    const int i = C.center;
    LQres f = lq(E, C.t[i], {0}, {1, 2});
    C.t[i] = f.Q;
    C.t[i - 1] = ein(E, "lpk,kr->lpr", C.t[i - 1], f.L);
    C.center--;
  }
}

DiagEnv vproduct(VTarget& g) {   // _variational_product
  DiagEnv C;
  for (const Par& p : g.single) {
    Tensor v = identity_leg(g.n.E, p);
    Tensor u = v;
    u.legs = {g.n.triv, v.legs[0], g.n.triv};
    u.dims = {1, v.dims[0], 1};
    u.strides = {v.dims[0], 1, 1};
    C.t.push_back(u);
  }
  C.edges = g.L.edges;
  C.center = 0;
  return C;
}


// _variational_input_identity: the identity on the leg of the layer site
// that takes `edge` as an input
Tensor input_identity(VTarget& g, int edge) {
  for (size_t j = 0; j < g.L.sites.size(); ++j) {
    auto ports = g.n.ports(g.L.sites[j][0], g.L.sites[j][1]);
    for (int k = 0; k < 4; ++k)
      if (ports[k] == edge) return identity_leg(g.n.E, g.legs4[j][k]);
  }
  throw Error(SPS_ERR_ARGUMENT, "input edge missing from variational layer");
}

// _variational_warm_start (diagonal_variational.jl:238-301)
DiagEnv vwarm_start(VTarget& g) {
  Engine& E = g.n.E;
  if (g.input.t.empty()) return vproduct(g);
  DiagEnv C;
  C.t = g.input.t;
  C.edges = g.input.edges;
  C.center = std::max(g.input.center, 0);
  std::vector<int> coords, oldc;
  for (int e : g.L.edges) coords.push_back(coordinate(g.n, e));
  for (int e : C.edges) oldc.push_back(coordinate(g.n, e));
  auto has = [&](int c) { return std::find(coords.begin(), coords.end(), c) != coords.end(); };
  // an end edge that leaves the frontier is capped with the identity
  while (!C.t.empty() && !has(oldc.front())) {
    vmove_center(E, C, 0);
    Tensor h = ein(E, "pr,p->r", drop_trivial(C.t[0], 0), input_identity(g, C.edges[0]));
    C.t.erase(C.t.begin());
    C.edges.erase(C.edges.begin());
    oldc.erase(oldc.begin());
    if (C.t.empty()) break;
    C.t[0] = with_trivial(ein(E, "r,rps->ps", h, C.t[0]), 1, true, g.n.triv);
    C.center = 0;
  }
  while (!C.t.empty() && !has(oldc.back())) {
    vmove_center(E, C, (int)C.t.size() - 1);
    Tensor h = ein(E, "lp,p->l", drop_trivial(C.t.back(), 2), input_identity(g, C.edges.back()));
    C.t.pop_back();
    C.edges.pop_back();
    oldc.pop_back();
    if (C.t.empty()) break;
    C.t.back() = with_trivial(ein(E, "lpr,r->lp", C.t.back(), h), 1, false, g.n.triv);
    C.center = (int)C.t.size() - 1;
  }
  if (C.t.empty()) return vproduct(g);
  // physical maps: embeddings keep the canonical form, projections first
  // move the centre there
  for (int i = 0; i < (int)C.t.size(); ++i) {
    const int j = (int)(std::find(coords.begin(), coords.end(), oldc[i]) - coords.begin());
    if (j >= (int)coords.size()) throw Error(SPS_ERR_ARGUMENT, "variational warm start: frontier edge not matched");
    const Par& P = C.t[i].legs[1];
    const Par& Q = g.physical[j];
    if (*P == *Q) continue;
    bool projects = false;
    for (int c = 0; c < 2; ++c) projects |= par_count(P, c) > par_count(Q, c);
    if (projects) vmove_center(E, C, i);
    const int nq = (int)Q->size(), np = (int)P->size();
    std::vector<double> mm((size_t)nq * np, 0.0);
    for (int c = 0; c < 2; ++c) {
      std::vector<int> qi, pi;
      for (int k = 0; k < nq; ++k)
        if ((*Q)[k] == c) qi.push_back(k);
      for (int k = 0; k < np; ++k)
        if ((*P)[k] == c) pi.push_back(k);
      for (size_t k = 0; k < std::min(qi.size(), pi.size()); ++k) mm[(size_t)qi[k] * np + pi[k]] = 1.0;
    }
    C.t[i] = ein(E, "qp,lpr->lqr", E.upload({Q, P}, mm.data()), C.t[i]);
  }
  DiagEnv product = vproduct(g);
  while (oldc.front() > coords.front()) {
    const int j = (int)(std::find(coords.begin(), coords.end(), oldc.front()) - coords.begin()) - 1;
    if (j < 0 || j >= (int)coords.size()) throw Error(SPS_ERR_ARGUMENT, "variational warm start: frontier edge not matched");
    C.t.insert(C.t.begin(), product.t[j]);
    oldc.insert(oldc.begin(), coords[j]);
    C.center++;
  }
  while (oldc.back() < coords.back()) {
    const int j = (int)(std::find(coords.begin(), coords.end(), oldc.back()) - coords.begin()) + 1;
    if (j <= 0 || j >= (int)coords.size()) throw Error(SPS_ERR_ARGUMENT, "variational warm start: frontier edge not matched");
    C.t.push_back(product.t[j]);
    oldc.push_back(coords[j]);
  }
  C.edges = g.L.edges;
  C.t[C.center] = contiguous(E, C.t[C.center]);
  const double s = norm(E, C.t[C.center]);
  if (s == 0) return product;
  if (!std::isfinite(s)) throw Error(SPS_ERR_NUMERIC, "nonfinite variational warm start");
  C.t[C.center] = clone(E, C.t[C.center]);
  scale_inplace(E, C.t[C.center], 1.0 / s);
  return C;
}

double nonnegative_residual(double value, double scale) {
  if (!std::isfinite(value)) throw VFail("nonfinite_residual");
  if (!(value >= -512 * DBL_EPSILON * std::max(1.0, scale))) throw VFail("negative_residual");
  return std::max(0.0, value);
}

// _variational_overlap_residual: |C - T|^2 with |T| = 1
double overlap_residual(VTarget& g, const DiagEnv& C, bool left, const VMsg* terminal) {
  VMsg term;
  if (terminal) {
    term = *terminal;
  } else {
    const int nc = (int)C.t.size();
    term = vedge(g, nc, left);
    for (int q = 0; q < nc; ++q) {
      const int i = left ? q : nc - 1 - q;
      term = vstep(g, term, i, C.t[i], left);
    }
  }
  VMsg edge = vedge(g, (int)C.t.size(), !left);
  LT v = join(g.n, term.m, edge.m);
  if (!v.number) throw Error(SPS_ERR_ARGUMENT, "unclosed variational overlap");
  const double overlap = v.s * std::exp(term.ls + edge.ls);
  const double nc = norm(g.n.E, C.t[C.center]);
  const double norm2 = nc * nc;
  if (!(std::isfinite(overlap) && std::isfinite(norm2))) throw VFail("nonfinite_overlap");
  return nonnegative_residual(1 + norm2 - 2 * overlap, std::max(norm2, 2 * std::fabs(overlap)));
}

struct HalfOut {
  double maxdiscard = 0, norm2 = 0;
  std::vector<VMsg> next;
};

// _variational_half_sweep! (diagonal_variational.jl:470-499)
HalfOut vhalf_sweep(VTarget& g, DiagEnv& C, const BMPS& m, bool right, Entropy* ent, std::vector<double>& profile,
                    const std::vector<VMsg>& fixed) {
  Engine& E = g.n.E;
  const int nc = (int)C.t.size();
  HalfOut out;
  VMsg rolling = vedge(g, nc, right);
  out.next.assign(nc + 1, VMsg());
  out.next[right ? 0 : nc] = rolling;
  Trunc tr;
  tr.chi = m.chi;
  tr.space[0] = m.space[0];
  tr.space[1] = m.space[1];
  std::vector<double> last;
  for (int q = 0; q + 1 < nc; ++q) {
    const int i = right ? q : nc - 2 - q;
    const VMsg& L = right ? rolling : fixed[i];
    const VMsg& R = right ? fixed[i + 2] : rolling;
    Tensor M = vpair(g, i, L, R);
    SVDres f = svd(E, M, {0, 1}, {2, 3}, tr, ent != nullptr);
    if (ent) {
      ent->maximum = std::max(ent->maximum, f.entropy);
      profile[i] = f.entropy;
    }
    if (f.norm == 0) throw VFail("zero_local_projection");
    last = f.S[0];
    last.insert(last.end(), f.S[1].begin(), f.S[1].end());
    out.maxdiscard = std::max(out.maxdiscard, (f.err / f.norm) * (f.err / f.norm));
    if (right) {
      C.t[i] = f.U;
      C.t[i + 1] = scale_leg(E, f.V, 0, last);
    } else {
      C.t[i] = scale_leg(E, f.U, 2, last);
      C.t[i + 1] = f.V;
    }
    C.center = right ? i + 1 : i;
    const int k = right ? i : i + 1;
    rolling = vstep(g, rolling, k, C.t[k], right);
    out.next[right ? k + 1 : k] = rolling;
  }
  for (double v : last) out.norm2 += v * v;
  if (out.norm2 == 0) throw VFail("zero_local_projection");
  return out;
}

// _variational_fit (diagonal_variational.jl:501-539)
DiagEnv vfit(VTarget& g, const BMPS& m, Entropy* ent, VariationalRecord& rec, std::vector<double>& bestprofile) {
  DiagEnv C = vwarm_start(g);
  const int nc = (int)C.t.size();
  const bool right = C.center < nc - 1 - C.center || (C.center == nc - 1 - C.center && !g.reverse);
  vmove_center(g.n.E, C, right ? 0 : nc - 1);
  std::vector<VMsg> fixed = vmessages(g, C, !right);
  const double initial = overlap_residual(g, C, !right, &fixed[right ? 0 : nc]);
  DiagEnv best = C;
  double cost = initial, change = INFINITY, discard = 0, previous = NAN;
  bestprofile.assign(std::max(0, nc - 1), NAN);
  int reason = VariationalRecord::SWEEP_LIMIT, sweeps = 0;
  for (int sweep = 1; sweep <= m.max_sweep; ++sweep) {
    std::vector<double> profile(nc - 1, NAN);
    sweeps = sweep;
    double current = INFINITY;
    std::string failure;
    try {
      HalfOut a = vhalf_sweep(g, C, m, right, ent, profile, fixed);
      HalfOut b = vhalf_sweep(g, C, m, !right, ent, profile, a.next);
      fixed = b.next;
      discard = std::max(discard, std::max(a.maxdiscard, b.maxdiscard));
      if (!(std::isfinite(b.norm2) && b.norm2 >= 0)) throw VFail("nonfinite_norm");
      current = nonnegative_residual(1 - b.norm2, b.norm2);
      if (!(current <= cost + 512 * DBL_EPSILON * std::max(1.0, cost))) throw VFail("residual_increase");
      change = sweep == 1 ? INFINITY : std::fabs(b.norm2 - previous) / std::max({b.norm2, previous, DBL_MIN});
      previous = b.norm2;
    } catch (const VFail& ex) {
      failure = ex.reason;
    } catch (const Error& ex) {
      if (ex.code != SPS_ERR_CONVERGENCE) throw;
      failure = "factorization_failure";
    }
    if (!failure.empty()) {
      rec.fallback = true;
      rec.fallback_reason = failure;
      reason = VariationalRecord::NUMERICAL_FALLBACK;
      break;
    }
    if (current <= cost) {
      best = C;
      cost = current;
      bestprofile = profile;
    }
    if (sweep > 1 && m.threshold_sweep > 0 && change <= m.threshold_sweep) {
      reason = VariationalRecord::THRESHOLD_SWEEP;
      break;
    }
  }
  rec.sweeps = sweeps;
  rec.relative_change = change;
  rec.stop_reason = reason;
  rec.initial_residual = initial;
  rec.residual = cost;
  rec.max_local_discarded_weight = discard;
  return best;
}

// _diagonal_absorb_layer! for the variational method (diagonal_variational.jl:541-614)
template <class Site>
void absorb_layer_variational(Net& n, DiagEnv& env, Site site, int t, const BMPS& m, bool reverse, Entropy* ent) {
  Engine& E = n.E;
  if (m.chi < 1) throw Error(SPS_ERR_ARGUMENT, "chi must be positive");
  if (m.max_sweep < 1) throw Error(SPS_ERR_ARGUMENT, "max_sweep must be positive");
  VTarget g = make_target(n, env, site, t, reverse);
  const int ne = (int)g.L.edges.size();
  std::vector<double> profile(std::max(0, ne - 1), NAN);
  VariationalRecord rec;
  rec.layer = t;
  rec.reverse = reverse;
  DiagEnv C;
  bool have = true;
  if (g.log_scale == -INFINITY) {
    if (ne == 0) {
      C.scalar = 0;
    } else {
      C = vproduct(g);
      C.t[C.center] = clone(E, C.t[C.center]);
      scale_inplace(E, C.t[C.center], 0.0);
    }
    rec.stop_reason = VariationalRecord::ZERO_TARGET;
    rec.residual = rec.initial_residual = NAN;
  } else if (ne <= 1) {
    if (ne == 0) {
      if (g.blocks.size() != 1 || g.blocks[0].size() != 1) throw Error(SPS_ERR_ARGUMENT, "diagonal corner is not closed");
      C.scalar = sum_all(E, g.blocks[0]);
    } else {
      C.t = {g.blocks[0]};
      C.edges = g.L.edges;
      C.center = 0;
    }
  } else if (g.L.sites.size() == 1) {
    Trunc tr;
    tr.chi = m.chi;
    tr.space[0] = m.space[0];
    tr.space[1] = m.space[1];
    SVDres f = svd(E, g.blocks[0], {0, 1}, {2, 3}, tr, ent != nullptr);
    if (ent) {
      ent->maximum = std::max(ent->maximum, f.entropy);
      profile[0] = f.entropy;
    }
    std::vector<double> sv(f.S[0]);
    sv.insert(sv.end(), f.S[1].begin(), f.S[1].end());
    C.t = {f.U, scale_leg(E, f.V, 0, sv)};
    C.edges = g.L.edges;
    C.center = 1;
    rec.residual = rec.max_local_discarded_weight = f.err * f.err;
  } else {
    try {
      C = vfit(g, m, ent, rec, profile);
    } catch (const VFail& ex) {
      have = false;
      rec.stop_reason = VariationalRecord::NUMERICAL_FALLBACK;
      rec.initial_residual = NAN;
      rec.residual = INFINITY;
      rec.fallback = true;
      rec.fallback_reason = ex.reason;
    }
    if (rec.fallback) {   // _variational_recover: the SVD absorption of the same layer
      DiagEnv alt = env;
      alt.max_trunc = 0;
      alt.variational.clear();
      BMPS plain = m;
      plain.variational = false;
      absorb_layer(n, alt, site, t, plain, reverse, nullptr);
      alt.t[alt.center] = clone(E, alt.t[alt.center]);
      scale_inplace(E, alt.t[alt.center], std::exp(alt.log_scale - g.log_scale));
      const double cost = overlap_residual(g, alt, true, nullptr);
      if (!std::isfinite(cost)) throw VFail("failed_svd_fallback");
      const bool use_svd = !have || cost < rec.residual;
      if (use_svd) {
        C = alt;
        rec.residual = cost;
      }
      rec.max_local_discarded_weight = std::max(rec.max_local_discarded_weight, alt.max_trunc);
      rec.used_svd = use_svd;
    }
  }
  double scale = 1.0;
  if (ne > 0) {
    C.t[C.center] = contiguous(E, C.t[C.center]);
    scale = norm(E, C.t[C.center]);
    if (!std::isfinite(scale)) throw Error(SPS_ERR_NUMERIC, "nonfinite variational boundary norm");
    if (scale != 0) {
      C.t[C.center] = clone(E, C.t[C.center]);
      scale_inplace(E, C.t[C.center], 1.0 / scale);
    }
  }
  std::vector<VariationalRecord> records = env.variational;
  records.push_back(rec);
  const double mt = std::isnan(rec.residual) ? env.max_trunc : std::max(env.max_trunc, rec.residual);
  env.t = C.t;
  env.edges = C.edges;
  env.center = C.center;
  env.scalar = C.scalar;
  env.log_scale = scale == 0 ? -INFINITY : g.log_scale + std::log(scale);
  env.max_trunc = mt;
  env.variational = records;
}

}  // namespace

// lognorm for the diagonal method (diagonal_mps.jl:315-323)
LogNorm lognorm_diagonal(Engine& E, const State& s, const BMPS& m) {
  Net n(E, s.Lx, s.Ly);
  DiagEnv env;
  auto site = [&](int x, int y) -> const Tensor& { return s.at(x, y); };
  for (int t = 0; t < s.Lx + s.Ly - 1; ++t) absorb_layer(n, env, site, t, m, false, nullptr);
  const double v = std::log(positive_real(env.scalar, "norm")) + env.log_scale;
  return {v + 2 * s.log_amplitude, v, env.max_trunc, env.variational};
}

// _diagonal_boundaries(side = :southeast) (diagonal_mps.jl:298-314)
void diagonal_southeast(Engine& E, const State& s, const BMPS& m, std::vector<DiagEnv>& se) {
  Net n(E, s.Lx, s.Ly);
  const int nl = s.Lx + s.Ly - 1;
  se.assign(nl + 1, DiagEnv());
  auto site = [&](int x, int y) -> const Tensor& { return s.at(x, y); };
  for (int t = nl - 1; t >= 0; --t) {
    se[t] = se[t + 1];
    absorb_layer(n, se[t], site, t, m, true, nullptr);
  }
}

std::vector<int> diagonal_draw_order(int Lx, int Ly) {
  std::vector<int> out;
  for (int t = 0; t < Lx + Ly - 1; ++t) {
    auto s = layer_sites(Lx, Ly, t);
    if (t % 2 == 1) std::reverse(s.begin(), s.end());
    for (auto& p : s) out.push_back(p[0] + p[1] * Lx);
  }
  return out;
}

}  // namespace sps

namespace sps {
namespace {

// DiagonalStrip / _diagonal_strip (diagonal_mps.jl:325-363): the sites of
// layers first..last by increasing x - y, the frontier tensors of the two
// boundaries attached to the site that owns their edge, unit vectors on
// open-boundary ports, and the unit ends of the boundary chains
struct Strip {
  std::vector<std::array<int, 2>> sites;
  std::vector<std::array<int, 4>> ports;
  std::vector<std::vector<LT>> att;
  LT left, right;
  double max_trunc = 0;
};

Strip make_strip(Net& n, int first, int last, const DiagEnv& nw, const DiagEnv& se) {
  Strip s;
  for (int t = first; t <= last; ++t)
    for (auto& p : layer_sites(n.Lx, n.Ly, t)) s.sites.push_back(p);
  std::stable_sort(s.sites.begin(), s.sites.end(),
                   [](const std::array<int, 2>& a, const std::array<int, 2>& b) { return a[0] - a[1] < b[0] - b[1]; });
  for (auto& p : s.sites) s.ports.push_back(n.ports(p[0], p[1]));
  s.att.resize(s.sites.size());
  s.left = number(1.0);
  s.right = number(1.0);
  int base = BOND;
  for (const DiagEnv* b : {&nw, &se}) {
    if (b->t.empty()) continue;
    if (b->t.front().dims[0] != 1 || b->t.back().dims[2] != 1)
      throw Error(SPS_ERR_ARGUMENT, "diagonal boundary ends are not trivial");
    const int len = (int)b->t.size();
    s.left = join(n, s.left, n.unit(base));
    s.right = join(n, s.right, n.unit(base + len));
    for (int k = 0; k < len; ++k) {
      const int edge = b->edges[k];
      int owner = -1;
      for (int i = 0; i < (int)s.ports.size() && owner < 0; ++i)
        if (std::find(s.ports[i].begin(), s.ports[i].end(), edge) != s.ports[i].end()) owner = i;
      if (owner < 0) throw Error(SPS_ERR_ARGUMENT, "boundary edge and diagonal strip are disconnected");
      s.att[owner].push_back(labelled(b->t[k], {base + k, edge, base + k + 1}));
    }
    base += len + 1;
  }
  for (size_t i = 0; i < s.sites.size(); ++i) {
    auto inside = n.inside(s.sites[i][0], s.sites[i][1]);
    for (int j = 0; j < 4; ++j)
      if (!inside[j]) s.att[i].push_back(n.unit(s.ports[i][j]));
  }
  s.max_trunc = std::max(nw.max_trunc, se.max_trunc);
  return s;
}

int shared(const LT& a, const LT& b) {
  int c = 0;
  for (int k : a.lab) c += index_of(b.lab, k) >= 0;
  return c;
}

// _diagonal_attach (diagonal_mps.jl:366-378): the pending tensor sharing the
// most labels (the first on ties); with none shared, the first unit vector
LT attach(Net& n, const LT& msg, std::vector<LT>& pending) {
  int best = 0, score = -1;
  for (int i = 0; i < (int)pending.size(); ++i) {
    const int c = shared(msg, pending[i]);
    if (c > score) {
      score = c;
      best = i;
    }
  }
  if (score == 0) {
    best = -1;
    for (int i = 0; i < (int)pending.size() && best < 0; ++i)
      if (pending[i].lab.size() == 1) best = i;
    if (best < 0) throw Error(SPS_ERR_ARGUMENT, "disconnected diagonal strip attachment");
  }
  LT a = pending[best];
  pending.erase(pending.begin() + best);
  return join(n, msg, a);
}

// _diagonal_step (diagonal_mps.jl:380-394)
LT step(Net& n, LT msg, const Strip& s, int k, const Tensor& A, const Tensor& B, const int* phys = nullptr) {
  std::vector<LT> pending = s.att[k];
  const auto& ports = s.ports[k];
  auto present = [&](const LT& m) {
    int c = 0;
    for (int p : ports) c += index_of(m.lab, p) >= 0;
    return c;
  };
  while (present(msg) < 2) {
    if (pending.empty()) throw Error(SPS_ERR_ARGUMENT, "missing diagonal strip inputs");
    msg = attach(n, msg, pending);
  }
  std::vector<int> inputs;
  for (int p : ports)
    if (index_of(msg.lab, p) >= 0) inputs.push_back(p);
  if (inputs.size() != 2) throw Error(SPS_ERR_ARGUMENT, "diagonal strip step has more than two inputs");
  msg = apply(n, msg, A, B, ports, inputs, phys);
  while (!pending.empty()) msg = attach(n, msg, pending);
  return msg;
}

// _diagonal_scale: divide by the norm on the device (a step's result owns its buffer)
LT scaled(Net& n, LT m) {
  if (m.number) {
    if (!std::isfinite(m.s)) throw Error(SPS_ERR_NUMERIC, "nonfinite diagonal environment");
    if (m.s != 0) m.s = m.s > 0 ? 1.0 : -1.0;
    return m;
  }
  safe_scale_inplace(n.E, m.t);
  m.unit = false;
  return m;
}

template <class Site>
void messages(Net& n, const Strip& s, Site site, int side /*0 both, 1 left, 2 right*/, std::vector<LT>& le,
              std::vector<LT>& ri) {
  const int m = (int)s.sites.size();
  le.assign(m + 1, LT());
  ri.assign(m + 1, LT());
  le[0] = s.left;
  ri[m] = s.right;
  if (side != 2)
    for (int k = 0; k < m; ++k) {
      const Tensor& A = site(s.sites[k][0], s.sites[k][1]);
      le[k + 1] = scaled(n, step(n, le[k], s, k, A, A));
    }
  if (side != 1)
    for (int k = m - 1; k >= 0; --k) {
      const Tensor& A = site(s.sites[k][0], s.sites[k][1]);
      ri[k] = scaled(n, step(n, ri[k + 1], s, k, A, A));
    }
}

double value(Net& n, const LT& l, const LT& r) {
  LT v = join(n, l, r);
  if (!v.number) throw Error(SPS_ERR_ARGUMENT, "unclosed diagonal network");
  return v.s;
}

// _diagonal_hole (diagonal_mps.jl:415-433): the attachments of the given
// sites joined to whichever half shares more labels, then the halves; legs
// in `output` order
Tensor hole(Net& n, LT left, LT right, const Strip& s, const std::vector<int>& positions,
            const std::vector<int>& output) {
  std::vector<LT> pending;
  for (int k : positions) pending.insert(pending.end(), s.att[k].begin(), s.att[k].end());
  while (!pending.empty()) {
    int li = 0, ri = 0, ls = -1, rs = -1;
    for (int i = 0; i < (int)pending.size(); ++i) {
      const int a = shared(left, pending[i]), b = shared(right, pending[i]);
      if (a > ls) {
        ls = a;
        li = i;
      }
      if (b > rs) {
        rs = b;
        ri = i;
      }
    }
    const bool useleft = ls > rs || (ls == rs && left.lab.size() <= right.lab.size());
    const int idx = useleft ? li : ri;
    LT a = pending[idx];
    pending.erase(pending.begin() + idx);
    if (useleft) left = join(n, left, a);
    else right = join(n, right, a);
  }
  return contiguous(n.E, reordered(join(n, left, right), output));
}

struct SiteRef {
  const State& s;
  const Tensor& operator()(int x, int y) const { return s.at(x, y); }
};

}  // namespace

// sample_configuration for the diagonal method (diagonal_born.jl:24-97):
// sites are drawn layer by layer (even layers by increasing x, odd ones by
// decreasing x; uniforms[i] is the uniform of the i-th site drawn), each
// layer inside a strip between the projected northwest boundary and the
// cached southeast one, then absorbed into the northwest boundary (the
// physical kind skips the last layer)
SampleResult sample_diagonal(Engine& E, const SamplingCache& c, const double* uniforms, const int* configuration) {
  const State& st = *c.state_ref;
  const int Lx = c.Lx, Ly = c.Ly, L = Lx * Ly, nl = Lx + Ly - 1;
  const bool physical = c.kind == KIND_PHYSICAL;
  Net n(E, Lx, Ly);
  SampleResult res;
  res.config.assign(L, 0);
  double maxtr = c.southeast.empty() ? 0.0 : c.southeast[0].max_trunc;
  res.max_env_trunc = maxtr;
  if (configuration) {
    int charge = 0;
    for (int i = 0; i < L; ++i) {
      if (configuration[i] != 1 && configuration[i] != 2)
        throw Error(SPS_ERR_ARGUMENT, "configuration contains an unknown basis label");
      charge ^= (*st.sites[i].legs[2])[configuration[i] - 1];
    }
    if (physical && charge != c.target) {
      for (int i = 0; i < L; ++i) res.config[i] = configuration[i];
      res.log_probability = -INFINITY;
      return res;
    }
  }
  DiagEnv nw;
  std::vector<Tensor> projected(L);
  auto proj_site = [&](int x, int y) -> const Tensor& { return projected[x + y * Lx]; };
  double logp = 0;
  int prefix = 0, position = 0;
  for (int t = 0; t < nl; ++t) {
    Strip s = make_strip(n, t, t, nw, c.southeast[t + 1]);
    const bool rightward = t % 2 == 0;
    std::vector<LT> le, ri;
    messages(n, s, SiteRef{st}, rightward ? 2 : 1, le, ri);
    LT msg = rightward ? s.left : s.right;
    const int m = (int)s.sites.size();
    for (int q = 0; q < m; ++q) {
      const int k = rightward ? q : m - 1 - q;
      const int x = s.sites[k][0], y = s.sites[k][1], site = x + y * Lx;
      const Tensor& A = st.sites[site];
      const LT& left = rightward ? msg : le[k];
      const LT& right = rightward ? ri[k + 1] : msg;
      bool allowed[2] = {true, true};
      if (physical)
        for (int j = 0; j < 2; ++j) allowed[j] = position < L - 1 || (prefix ^ (*A.legs[2])[j]) == c.target;
      if (!allowed[0] && !allowed[1]) throw Error(SPS_ERR_BORN, "sampling prefix violates the total symmetry sector");
      const auto& kets = c.candidate_kets[site];
      double p[2];
      LT next[2];
      if (physical) {
        std::vector<int> out(s.ports[k].begin(), s.ports[k].end());
        Tensor H = hole(n, left, right, s, {k}, out);
        for (int i = 3; i >= 0; --i) {
          if (*H.legs[i] != *fused_par({A.legs[VAX[i]], A.legs[VAX[i]]}))
            throw Error(SPS_ERR_ARGUMENT, "diagonal site hole does not match the site's legs");
          H = split(E, H, i, {A.legs[VAX[i]], A.legs[VAX[i]]});
        }
        Tensor root = metric_root(E, H, res);
        double values[2] = {0, 0};
        for (int j = 0; j < 2; ++j) {
          if (!allowed[j]) continue;
          Tensor u = ein(E, "wnpaes,wnesz->paz", kets[j], root);
          values[j] = dot(E, u, u);
        }
        const double total = values[0] + values[1];
        if (!std::isfinite(total)) throw Error(SPS_ERR_NUMERIC, "nonfinite proposal weight");
        if (total == 0) {
          const int na = (int)allowed[0] + (int)allowed[1];
          for (int j = 0; j < 2; ++j) p[j] = allowed[j] ? 1.0 / na : 0.0;
          res.zero_proposals++;
        } else {
          for (int j = 0; j < 2; ++j) p[j] = values[j] / total;
        }
      } else {
        double raw[2];
        for (int j = 0; j < 2; ++j) {
          next[j] = step(n, left, s, k, kets[j], kets[j]);
          raw[j] = value(n, next[j], right);
        }
        const double scale = std::max(std::fabs(raw[0]), std::fabs(raw[1]));
        for (double z : raw)
          if (!(std::isfinite(z) && z >= -64 * DBL_EPSILON * scale))
            throw Error(SPS_ERR_BORN, "invalid Born conditional at (" + std::to_string(x + 1) + "," +
                                          std::to_string(y + 1) + "); increase chi_sampling");
        const double v0 = std::max(raw[0], 0.0), v1 = std::max(raw[1], 0.0), total = v0 + v1;
        if (!(total > 0))
          throw Error(SPS_ERR_BORN, "Born conditional has zero total mass at (" + std::to_string(x + 1) + "," +
                                        std::to_string(y + 1) + ")");
        p[0] = v0 / total;
        p[1] = v1 / total;
      }
      int j;
      if (configuration) {
        j = configuration[site] - 1;
      } else {
        std::vector<double> lm{p[0] > 0 ? std::log(p[0]) : -INFINITY, p[1] > 0 ? std::log(p[1]) : -INFINITY};
        j = categorical(lm, uniforms[position], &res.near_boundary);
      }
      res.config[site] = j + 1;
      res.conditionals.push_back(p[j]);
      ++position;
      if (p[j] == 0.0) {
        res.log_probability = -INFINITY;
        res.max_env_trunc = maxtr;
        return res;
      }
      logp += std::log(p[j]);
      projected[site] = kets[j];
      if (physical) prefix ^= (*A.legs[2])[j];
      // moving from the left, the chosen candidate's step is the next message
      msg = scaled(n, (!physical && rightward) ? next[j] : step(n, msg, s, k, kets[j], kets[j]));
    }
    if (!physical || t < nl - 1) {
      absorb_layer(n, nw, proj_site, t, c.method, false, nullptr);
      maxtr = std::max(maxtr, nw.max_trunc);
    }
  }
  E.check_flag("sample_configuration");
  res.log_probability = logp;
  res.max_env_trunc = maxtr;
  return res;
}

// measure_energy for the diagonal method (diagonal_energy.jl:12-45): one-site
// terms in single-layer strips, bonds from layer t to t+1 in two-layer
// strips (_diagonal_layer_bonds, diagonal_update.jl:54-59; the pair value
// of diagonal_energy.jl:1-10 steps both sites with the operator kets)
EnergyResult measure_energy_diagonal(Engine& E, const State& s, const Model& m, const BMPS& method,
                                     bool record_entropy) {
  const int Lx = s.Lx, Ly = s.Ly, L = Lx * Ly, nl = Lx + Ly - 1;
  Net n(E, Lx, Ly);
  EnergyResult out;
  out.entropy.profile = record_entropy;
  out.entropy.Lx = Lx;
  out.entropy.Ly = Ly;
  if (record_entropy) {
    out.entropy.northwest.assign(L, NAN);
    out.entropy.southeast.assign(L, NAN);
  }
  Entropy* ent = record_entropy ? &out.entropy : nullptr;
  std::vector<DiagEnv> nw(nl + 1), se(nl + 1);
  SiteRef site{s};
  for (int t = 0; t < nl; ++t) {
    nw[t + 1] = nw[t];
    absorb_layer(n, nw[t + 1], site, t, method, false, ent);
  }
  for (int t = nl - 1; t >= 0; --t) {
    se[t] = se[t + 1];
    absorb_layer(n, se[t], site, t, method, true, ent);
  }
  Par p2 = make_par(1, 1);
  double xo[4] = {1, 0, 0, -1};
  Tensor X = E.upload({p2, p2}, xo);
  Tensor F, G;
  operator_factors(E, F, G);
  out.site_x.assign(L, 0.0);
  double xsum = 0, zzsum = 0;
  for (int t = 0; t < nl; ++t) {
    Strip st = make_strip(n, t, t, nw[t], se[t + 1]);
    std::vector<LT> le, ri;
    messages(n, st, site, 0, le, ri);
    for (int k = 0; k < (int)st.sites.size(); ++k) {
      const int x = st.sites[k][0], y = st.sites[k][1];
      const Tensor& A = s.at(x, y);
      const double den = value(n, step(n, le[k], st, k, A, A), ri[k + 1]);
      Tensor XA = ein(E, "pu,wnuaes->wnpaes", X, A);
      const double num = value(n, step(n, le[k], st, k, XA, A), ri[k + 1]);
      const double r = real_ratio(num, den);
      out.site_x[x + y * Lx] = r;
      xsum += r;
    }
    if (t == nl - 1) continue;
    Strip pst = make_strip(n, t, t + 1, nw[t], se[t + 2]);
    messages(n, pst, site, 0, le, ri);
    for (int dir = 0; dir < 2; ++dir) {
      const bool horizontal = dir == 0;
      auto sites = layer_sites(Lx, Ly, t);
      if (t % 2 == 1) std::reverse(sites.begin(), sites.end());
      for (auto& a : sites) {
        const int bx = a[0] + (horizontal ? 1 : 0), by = a[1] + (horizontal ? 0 : 1);
        if (bx >= Lx || by >= Ly) continue;
        int ia = -1, ib = -1;
        for (int k = 0; k < (int)pst.sites.size(); ++k) {
          if (pst.sites[k] == a) ia = k;
          if (pst.sites[k][0] == bx && pst.sites[k][1] == by) ib = k;
        }
        if (ia < 0 || ib < 0 || std::abs(ia - ib) != 1) throw Error(SPS_ERR_ARGUMENT, "nonadjacent diagonal observable");
        const Tensor& A = s.at(a[0], a[1]);
        const Tensor& B = s.at(bx, by);
        Tensor Cop, Dop;
        operator_pair(E, A, B, F, G, horizontal, Cop, Dop);
        auto pair_value = [&](const Tensor& KA, const Tensor& KB) {
          LT msg = le[std::min(ia, ib)];
          for (int k = std::min(ia, ib); k <= std::max(ia, ib); ++k) {
            const bool first = k == ia;
            msg = step(n, msg, pst, k, first ? KA : KB, first ? A : B);
          }
          return value(n, msg, ri[std::max(ia, ib) + 1]);
        };
        const double num = pair_value(Cop, Dop);
        const double den = pair_value(A, B);
        zzsum += real_ratio(num, den);
      }
    }
  }
  E.check_flag("measure_energy");
  const DiagEnv& fin = nw[nl];
  const double lnv = std::log(positive_real(fin.scalar, "norm")) + fin.log_scale;
  double hx = m.h * xsum;
  if (!m.fields.empty()) {
    hx = 0;
    for (int i = 0; i < L; ++i) hx += m.fields[i] * out.site_x[i];
  }
  out.energy_total = -m.J * zzsum - hx;
  out.energy_per_site = out.energy_total / L;
  out.log_norm = lnv + 2 * s.log_amplitude;
  out.tensor_log_norm = lnv;
  out.max_env_trunc = std::max(fin.max_trunc, se[0].max_trunc);
  out.x_sum = xsum;
  out.zz_sum = zzsum;
  return out;
}

}  // namespace sps

// ---------------------------------------------------------------------------
// full-update bond environments on diagonal boundaries
// (src/evolution/diagonal_update.jl)
// ---------------------------------------------------------------------------
namespace sps {
namespace {

// _diagonal_external_axes (diagonal_update.jl:12): the exterior legs of the
// bond's two sites, in the order of the reduced pair's Q factors
const int EXT_H[2][3] = {{0, 1, 5}, {1, 4, 5}}, EXT_V[2][3] = {{0, 1, 4}, {0, 4, 5}};
const int KA = -31, BA = -32, KB = -33, BB = -34;   // open core legs (ket, bra) of the two sites

std::vector<std::array<int, 2>> draw_sites(int Lx, int Ly, int t, bool reverse) {
  auto s = layer_sites(Lx, Ly, t);
  if ((t % 2 == 1) != reverse) std::reverse(s.begin(), s.end());
  return s;
}

// _diagonal_core_site (diagonal_update.jl:32-38): Q (three exterior legs,
// auxiliary, core) as a site tensor (w, n, p, a, e, s) whose physical leg is
// the core leg and whose bond leg is trivial
Tensor core_site(Net& n, const Tensor& Q, bool horizontal, bool first) {
  const int* ax = (horizontal ? EXT_H : EXT_V)[first ? 0 : 1];
  int missing = -1;
  for (int v : VAX)
    if (v != ax[0] && v != ax[1] && v != ax[2]) missing = v;
  Tensor t = with_trivial(Q, 1, false, n.triv);   // (x1, x2, x3, aux, core, trivial)
  std::vector<int> order(6);
  for (int i = 0; i < 3; ++i) order[ax[i]] = i;
  order[2] = 4;
  order[3] = 3;
  order[missing] = 5;
  return contiguous(n.E, perm_view(t, order));
}

struct DiagBond {   // DiagonalBondEnvironment (diagonal_update.jl:1-20)
  const Strip* strip;
  const LT* left;
  const LT* right;
  int a, b;                      // strip positions of the bond's sites, a < b
  std::array<int, 2> first, second;
  bool horizontal;
};

// _reduced_metric(::DiagonalBondEnvironment) (diagonal_update.jl:39-52): each
// core site closed against its own half, the open core pairs joined;
// N[rb, sb, rk, sk]
Tensor diag_metric(Net& n, const DiagBond& d, const Tensor& Qa, const Tensor& Qb) {
  Tensor A = core_site(n, Qa, d.horizontal, true), B = core_site(n, Qb, d.horizontal, false);
  auto absorb = [&](const LT& msg, int k) {
    const bool isfirst = d.strip->sites[k] == d.first;
    const int phys[2] = {isfirst ? KA : KB, isfirst ? BA : BB};
    const Tensor& C = isfirst ? A : B;
    return step(n, msg, *d.strip, k, C, C, phys);
  };
  LT l = absorb(*d.left, d.a), r = absorb(*d.right, d.b);
  return contiguous(n.E, reordered(join(n, l, r), {BA, BB, KA, KB}));
}

// bond_hole(::DiagonalBondEnvironment) (diagonal_update.jl:21-29): the six
// exterior double legs, each split (ket, bra)
Tensor diag_bond_hole(Net& n, const DiagBond& d, const State& st) {
  const auto& ax = d.horizontal ? EXT_H : EXT_V;
  std::vector<int> output;
  std::vector<Par> outer;
  for (int k = 0; k < 2; ++k) {
    const auto& site = k == 0 ? d.first : d.second;
    auto ports = n.ports(site[0], site[1]);
    for (int i = 0; i < 3; ++i) {
      const int axis = ax[k][i];
      output.push_back(ports[std::find(VAX, VAX + 4, axis) - VAX]);
      outer.push_back(st.at(site[0], site[1]).legs[axis]);
    }
  }
  Tensor H = hole(n, *d.left, *d.right, *d.strip, {d.a, d.b}, output);
  for (int k = 5; k >= 0; --k) {
    if (*H.legs[k] != *fused_par({outer[k], outer[k]}))
      throw Error(SPS_ERR_ARGUMENT, "diagonal bond hole does not match the sites' legs");
    H = split(n.E, H, k, {outer[k], outer[k]});
  }
  return H;
}

}  // namespace

// _sweep! on diagonal boundaries (diagonal_update.jl:61-102): the bonds from
// layer t to t+1 are updated inside a strip of the two layers between the
// rolling boundary of the finished layers and the cached boundary of the
// others; the rolling boundary then absorbs the finished layer
void sweep_diagonal(Engine& E, State& s, const Model& m, double delta, int D, const FUOptions& o,
                    const BMPS& method, bool horizontal, bool reverse, const int space[2], Entropy* ent,
                    StepReport& rep, double& env_err, bool force_repair) {
  const int Lx = s.Lx, Ly = s.Ly, nl = Lx + Ly - 1;
  Net n(E, Lx, Ly);
  SiteRef site{s};
  std::vector<DiagEnv> nw(nl + 1), se(nl + 1);
  if (reverse) {
    for (int t = 0; t < nl; ++t) {
      nw[t + 1] = nw[t];
      absorb_layer(n, nw[t + 1], site, t, method, false, ent);
      env_err = std::max(env_err, nw[t + 1].max_trunc);
    }
  } else {
    for (int t = nl - 1; t >= 0; --t) {
      se[t] = se[t + 1];
      absorb_layer(n, se[t], site, t, method, true, ent);
      if (t <= nl - 2) env_err = std::max(env_err, se[t].max_trunc);
    }
  }
  DiagEnv rolling;
  for (int q = 0; q + 1 < nl; ++q) {
    const int t = reverse ? nl - 2 - q : q;
    Strip st = make_strip(n, t, t + 1, reverse ? nw[t] : rolling, reverse ? rolling : se[t + 2]);
    auto order = draw_sites(Lx, Ly, t, reverse);
    const bool rightward = order.size() < 2 ? !reverse : order.front()[0] < order.back()[0];
    std::vector<LT> le, ri;
    messages(n, st, site, rightward ? 2 : 1, le, ri);
    LT msg = rightward ? st.left : st.right;
    const int ns = (int)st.sites.size();
    int cursor = rightward ? 0 : ns - 1;
    for (const auto& i : order) {   // _diagonal_layer_bonds(l, t, direction; reverse)
      const std::array<int, 2> j{i[0] + (horizontal ? 1 : 0), i[1] + (horizontal ? 0 : 1)};
      if (j[0] >= Lx || j[1] >= Ly) continue;
      int pi = -1, pj = -1;
      for (int k = 0; k < ns; ++k) {
        if (st.sites[k] == i) pi = k;
        if (st.sites[k] == j) pj = k;
      }
      if (pi < 0 || pj < 0 || std::abs(pi - pj) != 1)
        throw Error(SPS_ERR_ARGUMENT, "bond sites must be adjacent in a diagonal strip");
      const int a = std::min(pi, pj), b = std::max(pi, pj);
      while (rightward ? cursor < a : cursor > b) {
        const Tensor& A = s.at(st.sites[cursor][0], st.sites[cursor][1]);
        msg = scaled(n, step(n, msg, st, cursor, A, A));
        cursor += rightward ? 1 : -1;
      }
      DiagBond d{&st, rightward ? &msg : &le[a], rightward ? &ri[b + 1] : &msg, a, b, i, j, horizontal};
      PairEnv env;
      env.horizontal = horizontal;
      env.metric = [&](const Tensor& Qa, const Tensor& Qb) { return diag_metric(n, d, Qa, Qb); };
      env.hole = [&]() { return diag_bond_hole(n, d, s); };
      Tensor gate = trotter_gate(E, m, Lx, Ly, i[0], i[1], j[0], j[1], delta);
      BondReport br = update_bond_env(E, s, i[0], i[1], j[0], j[1], gate, D, o, env, space, force_repair);
      br.max_env_trunc = st.max_trunc;
      record_bond(rep, br, o);
      for (int k = rightward ? a : b; rightward ? k <= b : k >= a; k += rightward ? 1 : -1) {
        const Tensor& A = s.at(st.sites[k][0], st.sites[k][1]);
        msg = scaled(n, step(n, msg, st, k, A, A));
      }
      cursor = rightward ? b + 1 : a - 1;
    }
    absorb_layer(n, rolling, site, reverse ? t + 1 : t, method, reverse, ent);
    env_err = std::max(env_err, rolling.max_trunc);
  }
}

}  // namespace sps
