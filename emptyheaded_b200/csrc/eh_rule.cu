// Rule-level entry: a conjunctive COUNT rule over one binary relation, given
// as data (atoms over numbered variables, an optional equality selection),
// is matched to the device plan that computes it.
//
// Reference: the query compiler parses a Datalog rule (DatalogParser), plans a
// GHD (QueryPlanner, QueryPlannerTest.scala:78-304) and emits the bag code
// (EHGenerator.scala:728-838) that the generated run_<i> calls.  A COUNT over
// a rule body is the number of assignments of its variables that satisfy
// every atom, whatever the attribute order or the bag decomposition chosen,
// and it does not change when variables are renamed.  So the executor does
// not need the plan: it recognises the body up to renaming of variables and
// runs the device plan with the same count.  Recognised bodies (travis.py:
// 17, 58, 200, 241, 388, 476; the atoms' order and the names are free):
//   triangle   E(a,b) E(b,c) E(a,c)
//   4-clique   E(a,b) E(b,c) E(a,c) E(a,d) E(b,d) E(c,d)
//   lollipop   triangle(a,b,c) E(a,x)
//   barbell    triangle(a,b,c) E(a,x) triangle(x,y,z)
//   4-clique + E(a,x), x = v          (FliqueSelAgg)
//   triangle(a,b,c) E(a,p) E(p,x) triangle(x,y,z), p = v   (BarbellSelAgg)
// Any other body, or atoms over more than one relation, is EH_ERR_UNSUPPORTED.
#include <algorithm>
#include <set>
#include <utility>
#include <vector>

#include "eh_internal.cuh"

namespace eh {

namespace {

struct Shape {
  int query;
  int n_vars;
  std::vector<std::pair<int, int>> atoms;
  int sel_var;  // -1: no selection
};

const std::vector<Shape>& shapes() {
  // variables: a=0 b=1 c=2 d=3 / x=3 y=4 z=5 / p=6
  static const std::vector<Shape> s = {
      {EH_QUERY_TRIANGLE, 3, {{0, 1}, {1, 2}, {0, 2}}, -1},
      {EH_QUERY_CLIQUE4, 4, {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}}, -1},
      {EH_QUERY_LOLLIPOP, 4, {{0, 1}, {1, 2}, {0, 2}, {0, 3}}, -1},
      {EH_QUERY_BARBELL, 6, {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {3, 4}, {4, 5}, {3, 5}}, -1},
      {EH_QUERY_CLIQUE4_SEL, 5, {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}, {0, 4}}, 4},
      {EH_QUERY_BARBELL_SEL, 7, {{0, 1}, {1, 2}, {0, 2}, {0, 6}, {6, 3}, {3, 4}, {4, 5}, {3, 5}}, 6},
  };
  return s;
}

// is there a renaming of the rule's variables onto the shape's with the same
// atom set (and the selected variable onto the shape's)?
bool matches(const Shape& sh, int n_vars, const std::set<std::pair<int, int>>& atoms, int sel) {
  if (n_vars != sh.n_vars || atoms.size() != sh.atoms.size() || (sel >= 0) != (sh.sel_var >= 0)) return false;
  std::set<std::pair<int, int>> want(sh.atoms.begin(), sh.atoms.end());
  std::vector<int> perm(n_vars);
  for (int i = 0; i < n_vars; i++) perm[i] = i;
  do {  // at most 7! renamings
    if (sel >= 0 && perm[sel] != sh.sel_var) continue;
    bool ok = true;
    for (const auto& a : atoms)
      if (!want.count({perm[a.first], perm[a.second]})) {
        ok = false;
        break;
      }
    if (ok) return true;
  } while (std::next_permutation(perm.begin(), perm.end()));
  return false;
}

}  // namespace

int rule_match(const eh_rule* rule, uint32_t* relation) {
  EH_REQUIRE(rule && (rule->n_atoms == 0 || rule->atoms), EH_ERR_INVALID, "null rule");
  EH_REQUIRE(rule->n_vars >= 1 && rule->n_vars <= 7, EH_ERR_UNSUPPORTED,
             "rules with more than 7 variables are not planned on the device");
  EH_REQUIRE(rule->sel_var < (int32_t)rule->n_vars, EH_ERR_INVALID, "selected variable out of range");
  std::set<std::pair<int, int>> atoms;
  std::vector<bool> used(rule->n_vars, false);
  uint32_t rel = 0;
  for (uint32_t i = 0; i < rule->n_atoms; i++) {
    const eh_atom& a = rule->atoms[i];
    EH_REQUIRE(a.v0 < rule->n_vars && a.v1 < rule->n_vars, EH_ERR_INVALID, "atom variable out of range");
    if (i == 0) rel = a.relation;
    EH_REQUIRE(a.relation == rel, EH_ERR_UNSUPPORTED, "rules over more than one relation are not planned");
    EH_REQUIRE(a.v0 != a.v1, EH_ERR_UNSUPPORTED, "atoms with a repeated variable are not planned");
    atoms.insert({(int)a.v0, (int)a.v1});  // a repeated atom is the same constraint
    used[a.v0] = used[a.v1] = true;
  }
  for (uint32_t v = 0; v < rule->n_vars; v++)
    EH_REQUIRE(used[v], EH_ERR_UNSUPPORTED, "every variable must appear in an atom");
  for (const Shape& sh : shapes())
    if (matches(sh, (int)rule->n_vars, atoms, rule->sel_var)) {
      if (relation) *relation = rel;
      return sh.query;
    }
  throw Error{EH_ERR_UNSUPPORTED, "rule body is none of the device plans (triangle, 4-clique, lollipop, barbell, "
                                  "4-clique or barbell with a selection)"};
}

}  // namespace eh
