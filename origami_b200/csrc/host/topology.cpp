// Bonded topology graph: restates geom/src/topology_graph.rs:134-389.
//
// Bond sources, in the reference's order of discovery (a set, so order does
// not matter): backbone N-CA, CA-C, C-O, N-H, CA-HA(2/3); the peptide bond
// C(i-1)-N(i) inside one chain; side-chain template bond_to parents; ring
// closures (Pro N-CD, Phe/Tyr CE2-CZ, His CE1-NE2, Trp CE2-CD2 and CH2-CZ3);
// disulfides between Cys SG atoms within 2.5 A.  Bonds are sorted by (a, b);
// angles enumerate neighbour pairs per central atom; proper dihedrals walk the
// sorted bond list and keep first occurrences of the canonical (b < c) key;
// impropers are listed per residue (peptide C, Asn CG, Gln CD, Asp CG, Glu CD,
// Arg CZ).
#include <algorithm>
#include <map>
#include <queue>
#include <set>

#include "model.h"

namespace og {

namespace {
const std::vector<std::pair<const char*, const char*>>& ring_closures(int aa) {
  static const std::vector<std::pair<const char*, const char*>> none;
  static const std::vector<std::pair<const char*, const char*>> pro = {{"N", "CD"}};
  static const std::vector<std::pair<const char*, const char*>> phe = {{"CE2", "CZ"}};
  static const std::vector<std::pair<const char*, const char*>> his = {{"CE1", "NE2"}};
  static const std::vector<std::pair<const char*, const char*>> trp = {{"CE2", "CD2"}, {"CH2", "CZ3"}};
  switch (aa) {
    case PRO: return pro;
    case PHE: return phe;
    case TYR: return phe;
    case HIS: return his;
    case TRP: return trp;
    default: return none;
  }
}
}  // namespace

Topology build_topology(const Structure& s, const Templates& tpl) {
  std::map<std::pair<int, std::string>, int> idx;
  int total = 0;
  for (size_t ri = 0; ri < s.residues.size(); ++ri)
    for (const auto& a : s.residues[ri].atoms) idx[{static_cast<int>(ri), a.name}] = total++;
  auto lookup = [&](int ri, const std::string& name) -> int {
    auto it = idx.find({ri, name});
    return it == idx.end() ? -1 : it->second;
  };

  std::set<std::pair<int, int>> bondset;
  auto add_bond = [&](int a, int b) {
    if (a < 0 || b < 0 || a == b) return;
    bondset.insert(a < b ? std::make_pair(a, b) : std::make_pair(b, a));
  };

  for (size_t r = 0; r < s.residues.size(); ++r) {
    const int ri = static_cast<int>(r);
    const PlacedResidue& res = s.residues[r];
    const int aa = res.aa;
    int n = lookup(ri, "N"), ca = lookup(ri, "CA"), c = lookup(ri, "C"), o = lookup(ri, "O");
    add_bond(n, ca);
    add_bond(ca, c);
    add_bond(c, o);
    add_bond(n, lookup(ri, "H"));
    if (aa == GLY) {
      add_bond(ca, lookup(ri, "HA2"));
      add_bond(ca, lookup(ri, "HA3"));
    } else {
      add_bond(ca, lookup(ri, "HA"));
    }
    if (ri > 0 && s.residues[r - 1].chain == res.chain) add_bond(lookup(ri - 1, "C"), n);
    for (const TemplateAtom& sc : tpl.get(aa).sidechain) add_bond(lookup(ri, sc.bond_to), lookup(ri, sc.name));
    for (const auto& rc : ring_closures(aa)) add_bond(lookup(ri, rc.first), lookup(ri, rc.second));
  }

  // Disulfides: Cys SG pairs within 2.5 A.
  std::vector<std::pair<int, Vec3>> sg;
  for (size_t r = 0; r < s.residues.size(); ++r) {
    if (s.residues[r].aa != CYS) continue;
    for (const auto& a : s.residues[r].atoms)
      if (a.name == "SG") sg.push_back({lookup(static_cast<int>(r), "SG"), a.pos});
  }
  const double max_sq = 2.5 * 2.5;
  for (size_t i = 0; i < sg.size(); ++i)
    for (size_t j = i + 1; j < sg.size(); ++j) {
      Vec3 d{sg[i].second.x - sg[j].second.x, sg[i].second.y - sg[j].second.y,
             sg[i].second.z - sg[j].second.z};
      if (d.x * d.x + d.y * d.y + d.z * d.z <= max_sq) add_bond(sg[i].first, sg[j].first);
    }

  Topology t;
  for (const auto& b : bondset) t.bonds.push_back({b.first, b.second});  // std::set is (a, b)-sorted
  t.bonded_to.assign(total, {});
  for (const auto& b : t.bonds) {
    t.bonded_to[b[0]].push_back(b[1]);
    t.bonded_to[b[1]].push_back(b[0]);
  }
  for (auto& nb : t.bonded_to) std::sort(nb.begin(), nb.end());

  for (int b = 0; b < total; ++b) {
    const auto& nb = t.bonded_to[b];
    for (size_t i = 0; i < nb.size(); ++i)
      for (size_t j = i + 1; j < nb.size(); ++j) t.angles.push_back({nb[i], b, nb[j]});
  }

  std::set<std::array<int, 4>> seen;
  for (const auto& bond : t.bonds) {
    const int b = bond[0], c = bond[1];
    for (int a : t.bonded_to[b]) {
      if (a == c) continue;
      for (int d : t.bonded_to[c]) {
        if (d == b || d == a) continue;
        std::array<int, 4> key = b < c ? std::array<int, 4>{a, b, c, d} : std::array<int, 4>{d, c, b, a};
        if (seen.insert(key).second) t.dihedrals.push_back(key);
      }
    }
  }

  const int nres = static_cast<int>(s.residues.size());
  for (int ri = 0; ri < nres; ++ri) {
    const int aa = s.residues[ri].aa;
    if (ri + 1 < nres) {
      int ca = lookup(ri, "CA"), c = lookup(ri, "C"), o = lookup(ri, "O"), nn = lookup(ri + 1, "N");
      if (ca >= 0 && c >= 0 && o >= 0 && nn >= 0) t.impropers.push_back({c, ca, o, nn});
    }
    auto imp = [&](const char* sub0, const char* central, const char* sub1, const char* sub2) {
      int x0 = lookup(ri, sub0), xc = lookup(ri, central), x1 = lookup(ri, sub1), x2 = lookup(ri, sub2);
      if (x0 >= 0 && xc >= 0 && x1 >= 0 && x2 >= 0) t.impropers.push_back({xc, x0, x1, x2});
    };
    switch (aa) {
      case ASN: imp("CB", "CG", "OD1", "ND2"); break;
      case GLN: imp("CG", "CD", "OE1", "NE2"); break;
      case ASP: imp("CB", "CG", "OD1", "OD2"); break;
      case GLU: imp("CG", "CD", "OE1", "OE2"); break;
      case ARG: imp("NE", "CZ", "NH1", "NH2"); break;
      default: break;
    }
  }
  return t;
}

std::vector<ExclusionPair> build_exclusions(const Topology& t, int n_atoms) {
  // Graph distance 1 or 2 -> excluded, exactly 3 -> 1-4 (equivalent to the
  // is_bonded / is_one_three / is_one_four predicates, which test for walks
  // of length 1, 2 and 3).
  std::vector<ExclusionPair> out;
  std::vector<int> dist(n_atoms, -1);
  std::vector<int> touched;
  for (int i = 0; i < n_atoms; ++i) {
    touched.clear();
    std::queue<int> q;
    dist[i] = 0;
    touched.push_back(i);
    q.push(i);
    while (!q.empty()) {
      int u = q.front();
      q.pop();
      if (dist[u] == 3) continue;
      for (int v : t.bonded_to[u]) {
        if (dist[v] >= 0) continue;
        dist[v] = dist[u] + 1;
        touched.push_back(v);
        q.push(v);
      }
    }
    std::vector<ExclusionPair> row;
    for (int v : touched) {
      if (v <= i) continue;
      if (dist[v] == 1 || dist[v] == 2) row.push_back({i, v, 1});
      else if (dist[v] == 3) row.push_back({i, v, 2});
    }
    std::sort(row.begin(), row.end(), [](const ExclusionPair& a, const ExclusionPair& b) { return a.j < b.j; });
    out.insert(out.end(), row.begin(), row.end());
    for (int v : touched) dist[v] = -1;
  }
  return out;
}

}  // namespace og
