#include "geometry.h"

#include <algorithm>
#include <cmath>
#include <utility>

namespace artss {

// ------------------------------------------------------------------ merges

IdxList merge_keep(const IdxList &a, const IdxList &b) {
    // Algorithm::merge_sort (src/utility/Algorithm.cpp:22-54): ties take b
    IdxList out;
    out.reserve(a.size() + b.size());
    size_t p = 0, q = 0;
    while (p < a.size() && q < b.size()) out.push_back(a[p] < b[q] ? a[p++] : b[q++]);
    while (p < a.size()) out.push_back(a[p++]);
    while (q < b.size()) out.push_back(b[q++]);
    return out;
}

IdxList merge_unique(const IdxList &a, const IdxList &b) {
    // Algorithm::merge_sort_with_duplicates (src/utility/Algorithm.cpp:65-113)
    if (a.empty()) return b;
    if (b.empty()) return a;
    IdxList out;
    out.reserve(a.size() + b.size());
    size_t p = 0, q = 0;
    auto step = [&]() {
        if (a[p] < b[q]) out.push_back(a[p++]);
        else if (a[p] > b[q]) out.push_back(b[q++]);
        else { out.push_back(a[p]); p++; q++; }
    };
    step();
    while (p < a.size() && q < b.size()) step();
    if (p < a.size()) {
        if (a[p] == out.back()) p++;
        while (p < a.size()) out.push_back(a[p++]);
    } else if (q < b.size()) {
        if (b[q] == out.back()) q++;
        while (q < b.size()) out.push_back(b[q++]);
    }
    return out;
}

// ------------------------------------------------------------------ grid

Grid::Grid(const settings::Domain &d, size_t levels) : levels_(levels), lv_(levels + 1) {
    start_pd = d.start_PD;
    end_pd = d.end_PD;
    start_cd = d.start_CD;
    end_cd = d.end_CD;
    for (int a = 0; a < 3; a++) length_pd[a] = std::fabs(end_pd[a] - start_pd[a]);
    lv_[0].n = d.n;
    for (size_t l = 0; l <= levels; l++) {
        GridLevel &g = lv_[l];
        for (int a = 0; a < 3; a++) {
            if (l > 0) {
                const size_t prev = lv_[l - 1].n[a];
                g.n[a] = prev == 1 ? 1 : (size_t) std::round((double) (prev / 2));
            }
            if (g.n[a] == 0) throw config_error("number of inner cells must be positive");
            g.spacing[a] = length_cd(a) / (double) g.n[a];
            g.N[a] = (size_t) (std::round(length_pd[a] / g.spacing[a]) + 2);
            g.cd_start[a] = (size_t) std::round((start_cd[a] - start_pd[a]) / g.spacing[a]) + 1;
            g.cd_end[a] = (size_t) std::round((end_cd[a] - start_pd[a]) / g.spacing[a]);
            // The reference sizes its inner and boundary lists by the level's cell
            // count (Domain::init, src/domain/Domain.cpp:40-54) but fills them over
            // the index range above (Domain::inner_cells, Domain.cpp:191-203).  When a
            // computational domain's bounds fall between a coarse level's cells the
            // rounding makes the two differ by one: the reference then writes past
            // its lists or leaves zero entries in them.  Such a domain is refused.
            if (g.cd_end[a] + 1 < g.cd_start[a] || g.cd_end[a] + 1 - g.cd_start[a] != g.n[a])
                throw config_error("computational domain bounds fall between the cells of multigrid level " +
                                   std::to_string(l) + " on axis " + std::string(1, "xyz"[a]) + " (" +
                                   std::to_string(g.n[a]) + " cells, index range " + std::to_string(g.cd_start[a]) +
                                   ".." + std::to_string(g.cd_end[a]) + ")");
        }
    }
}

double Grid::length_cd(int axis) const { return std::fabs(end_cd[axis] - start_cd[axis]); }

// ------------------------------------------------------------------ obstacles

bool ObstacleBox::contains(double x, double y, double z) const {
    return (double) start[0] <= x && x <= (double) end[0] && (double) start[1] <= y && y <= (double) end[1] &&
           (double) start[2] <= z && z <= (double) end[2];
}

bool ObstacleBox::intersects(const std::array<size_t, 3> &source, const std::array<size_t, 3> &cell) const {
    const double eps = 10E-6;
    if (start[0] <= cell[0] && cell[0] <= end[0] && start[1] <= cell[1] && cell[1] <= end[1] && start[2] <= cell[2] &&
        cell[2] <= end[2])
        return true;
    double line0[3], line1[3], dir[3];
    for (int a = 0; a < 3; a++) {
        line0[a] = (double) source[a] + 0.5;
        line1[a] = (double) cell[a] + 0.5;
        dir[a] = line1[a] - line0[a];
    }
    for (int axis = 0; axis < 3; axis++) {
        double area0[3], area1[3];
        for (int a = 0; a < 3; a++) {
            area0[a] = (double) start[a] + 0.5;
            area1[a] = (double) end[a] + 0.5;
        }
        for (int patch = 2 * axis; patch <= 2 * axis + 1; patch++) {
            if (patch % 2 == 1) std::swap(area0, area1);
            // the patch normal is e_axis, so dot(normal, dir) == dir[axis]
            if (std::fabs(dir[axis]) > eps) {
                const double lambda = (area0[axis] - line0[axis]) / dir[axis];
                if (lambda <= 1 && lambda >= 0) {
                    double p[3];
                    for (int a = 0; a < 3; a++) p[a] = dir[a] * lambda + line0[a] - 0.5;
                    if (contains(p[0], p[1], p[2])) return true;
                }
            }
        }
    }
    return false;
}

namespace {

ObstacleBox make_box(const std::string &name, std::array<size_t, 3> start, std::array<size_t, 3> end,
                     const GridLevel &g) {
    // Obstacle::init / create_obstacle / remove_cells_at_boundary (src/domain/Obstacle.cpp:51-191, :458-478)
    ObstacleBox b;
    b.name = name;
    b.start = start;
    b.end = end;
    std::array<size_t, 3> s{};
    for (int a = 0; a < 3; a++) s[a] = end[a] - start[a] + 1;
    std::array<size_t, 6> size{};
    size[FRONT] = size[BACK] = s[1] * s[0];
    size[BOTTOM] = size[TOP] = s[2] * s[0];
    size[LEFT] = size[RIGHT] = s[2] * s[1];
    if (start[2] <= g.cd_start[2]) size[FRONT] = 0;
    if (end[2] >= g.cd_end[2]) size[BACK] = 0;
    if (start[1] <= g.cd_start[1]) size[BOTTOM] = 0;
    if (end[1] >= g.cd_end[1]) size[TOP] = 0;
    if (start[0] <= g.cd_start[0]) size[LEFT] = 0;
    if (end[0] >= g.cd_end[0]) size[RIGHT] = 0;
    b.cells.reserve(s[0] * s[1] * s[2]);
    for (size_t k = start[2]; k <= end[2]; k++)
        for (size_t j = start[1]; j <= end[1]; j++)
            for (size_t i = start[0]; i <= end[0]; i++) b.cells.push_back(g.index(i, j, k));
    auto face = [&](int p, int fixed_axis, size_t fixed, int outer, int inner) {
        if (size[p] == 0) return;
        IdxList &L = b.patch[p];
        L.reserve(size[p]);
        std::array<size_t, 3> c{};
        c[fixed_axis] = fixed;
        for (size_t o = start[outer]; o <= end[outer]; o++)
            for (size_t q = start[inner]; q <= end[inner]; q++) {
                c[outer] = o;
                c[inner] = q;
                L.push_back(g.index(c[0], c[1], c[2]));
            }
    };
    face(FRONT, 2, start[2], 1, 0);
    face(BACK, 2, end[2], 1, 0);
    face(BOTTOM, 1, start[1], 2, 0);
    face(TOP, 1, end[1], 2, 0);
    face(LEFT, 0, start[0], 2, 1);
    face(RIGHT, 0, end[0], 2, 1);
    return b;
}

bool overlap_1d(size_t a1, size_t a2, size_t b1, size_t b2) { return a1 <= b2 && a2 >= b1; }

// Obstacle::calculate_area_index (src/domain/Obstacle.cpp:513-544)
void area_index(const ObstacleBox &o1, const ObstacleBox &o2, size_t &c1, size_t &c2, int axis, bool start) {
    if (start) {
        c1 = o1.start[axis];
        c2 = o2.start[axis];
        if (o1.start[axis] > o2.start[axis]) c2 = o1.start[axis] + 1;
        else if (o1.start[axis] < o2.start[axis]) c1 = o2.start[axis] + 1;
    } else {
        c1 = o1.end[axis];
        c2 = o2.end[axis];
        if (o1.end[axis] < o2.end[axis]) c2 = o1.end[axis] - 1;
        else if (o1.end[axis] > o2.end[axis]) c1 = o2.end[axis] - 1;
    }
}

// One obstacle's side of the cell removal of Obstacle::circular_constraints
// (src/domain/Obstacle.cpp:700-808): the cells of the rectangle [rs, re]
// (fixed on `axis`) are removed from a sorted patch list by a cursor that
// moves over the rectangle in ascending order, and only on a match.  Cells
// below the rectangle's first cell are kept as they are; where every cell of
// the list lies below it, the reference reads on past the end of the list
// (Obstacle.cpp:704-723) and its result depends on the memory behind it, and
// this walk stops at the end.
struct PatchWalk {
    const IdxList &in;
    const GridLevel &g;
    std::array<size_t, 3> cur, re;
    size_t reset0;  // the cursor's first coordinate on the inner axis
    int o0, o1;
    size_t pos = 0;
    bool ended = false;
    Idx target;
    IdxList out;

    PatchWalk(const IdxList &list, const std::array<size_t, 3> &rs, const std::array<size_t, 3> &re_, int inner,
              int outer, const GridLevel &gl)
        : in(list), g(gl), cur(rs), re(re_), reset0(rs[inner]), o0(inner), o1(outer) {
        target = g.index(cur[0], cur[1], cur[2]);
        out.reserve(in.size());
        while (pos < in.size() && in[pos] < target) out.push_back(in[pos++]);
    }
    bool more() const { return pos < in.size(); }
    bool in_rows() const { return cur[o1] <= re[o1]; }
    void step() {
        const Idx e = in[pos++];
        if (e != target) {
            out.push_back(e);
            return;
        }
        if (++cur[o0] > re[o0]) {
            cur[o0] = reset0;
            if (++cur[o1] > re[o1]) ended = true;
        }
        target = g.index(cur[0], cur[1], cur[2]);
    }
};

// Both walks run in one loop (Obstacle.cpp:734-771) while both lists have
// cells and neither rectangle is exhausted; the walk left over then continues only while its
// cursor row lies inside its rectangle.  The coupling matters where
// calculate_area_index makes a rectangle empty on the outer axis (two
// obstacles side by side but offset): its first matching cell is removed
// only if the joint loop reaches it.
void remove_rects(IdxList &l1, IdxList &l2, const std::array<size_t, 3> &r1s, const std::array<size_t, 3> &r1e,
                  const std::array<size_t, 3> &r2s, const std::array<size_t, 3> &r2e, int inner, int outer,
                  const GridLevel &g) {
    PatchWalk w1(l1, r1s, r1e, inner, outer, g), w2(l2, r2s, r2e, inner, outer, g);
    while (w1.more() && w2.more() && !w1.ended && !w2.ended) {
        w1.step();
        w2.step();
    }
    for (PatchWalk *w : {&w1, &w2}) {
        if (!w->ended)
            while (w->more() && w->in_rows()) w->step();
        while (w->more()) w->out.push_back(w->in[w->pos++]);
    }
    l1 = std::move(w1.out);
    l2 = std::move(w2.out);
}

// Obstacle::circular_constraints (src/domain/Obstacle.cpp:597-859): o1 lies
// directly after o2 along `axis`
void circular_constraints(ObstacleBox &o1, ObstacleBox &o2, int axis, const GridLevel &g) {
    if (o1.start[axis] - 1 != o2.end[axis]) return;
    const int ax0 = axis == 0 ? 1 : 0;
    const int ax1 = axis == 2 ? 1 : 2;
    if (!(overlap_1d(o1.start[ax0], o1.end[ax0], o2.start[ax0], o2.end[ax0]) &&
          overlap_1d(o1.start[ax1], o1.end[ax1], o2.start[ax1], o2.end[ax1])))
        return;
    const int p1 = 2 * axis;      // LEFT / BOTTOM / FRONT of o1
    const int p2 = 2 * axis + 1;  // RIGHT / TOP / BACK of o2
    std::array<size_t, 3> r1s{}, r1e{}, r2s{}, r2e{};
    r1s[axis] = r1e[axis] = o1.start[axis];
    r2s[axis] = r2e[axis] = o2.end[axis];
    area_index(o1, o2, r1s[ax0], r2s[ax0], ax0, true);
    area_index(o1, o2, r1e[ax0], r2e[ax0], ax0, false);
    area_index(o1, o2, r1s[ax1], r2s[ax1], ax1, true);
    area_index(o1, o2, r1e[ax1], r2e[ax1], ax1, false);
    remove_rects(o1.patch[p1], o2.patch[p2], r1s, r1e, r2s, r2e, ax0, ax1, g);
}

void fill_bc(BcTable &t, const std::vector<settings::Boundary> &bs) {
    for (const auto &b : bs)
        for (int ft : b.field_types)
            for (int p : b.patches) {
                t[ft].present = true;
                t[ft].bc[p] = b.bc;
                t[ft].has_value[p] = b.value.has_value();
                t[ft].value[p] = b.value.value_or(0.0);
            }
}

void check_bc(const BcTable &t, const std::vector<settings::Boundary> &bs, const std::string &owner) {
    std::array<std::array<bool, 6>, 7> set{};
    for (const auto &b : bs)
        for (int ft : b.field_types)
            for (int p : b.patches) set[ft][p] = true;
    for (int ft = 0; ft < 7; ft++) {
        if (!t[ft].present) continue;
        for (int p = 0; p < 6; p++)
            if (!set[ft][p])
                throw config_error(owner + ": field '" + kFieldTypeNames[ft] + "' has no boundary condition on patch '" +
                                   kPatchNames[p] + "'");
    }
}

}  // namespace

// ------------------------------------------------------------------ geometry

Geometry::Geometry(const settings::Settings &s)
    : grid_(s.domain, s.solver.description.find("NS") != std::string::npos || s.solver.description == "PressureSolver"
                          ? s.solver.pressure.n_level
                          : 0) {
    const size_t L = grid_.levels();
    fill_bc(domain_bc_, s.boundaries);
    check_bc(domain_bc_, s.boundaries, "domain");

    // level-0 obstacles from physical coordinates (Obstacle.cpp:13-29)
    std::vector<ObstacleBox> lvl0;
    if (s.obstacles_enabled) {
        const GridLevel &g0 = grid_.level(0);
        for (const auto &o : s.obstacles) {
            std::array<size_t, 3> st{}, en{};
            for (int a = 0; a < 3; a++) {
                const double h = grid_.length_cd(a) / (double) g0.n[a];
                st[a] = (size_t) (static_cast<int>(std::round((-grid_.start_pd[a] + o.start[a]) / h)) + 1);
                en[a] = (size_t) static_cast<int>(std::round((-grid_.start_pd[a] + o.end[a]) / h));
                if (en[a] < st[a] || en[a] >= g0.N[a] - 1 || st[a] < 1)
                    throw config_error("obstacle '" + o.name + "' lies outside the domain or is thinner than a cell");
            }
            lvl0.push_back(make_box(o.name, st, en, g0));
            BcTable t{};
            fill_bc(t, o.boundaries);
            check_bc(t, o.boundaries, "obstacle '" + o.name + "'");
            obstacle_bc_.push_back(t);
        }
        // DomainController::detect_neighbouring_obstacles (src/domain/DomainController.cpp:154-173)
        for (size_t a = 0; a < lvl0.size(); a++)
            for (size_t b = a + 1; b < lvl0.size(); b++)
                for (int axis = 0; axis < 3; axis++) {
                    if (lvl0[a].end[axis] + 1 == lvl0[b].start[axis])
                        circular_constraints(lvl0[b], lvl0[a], axis, g0);
                    else
                        circular_constraints(lvl0[a], lvl0[b], axis, g0);
                }
    }

    // per-level obstacles and merged obstacle lists (Multigrid.cpp:180-265, :438-514)
    obstacles_.resize(L + 1);
    obstacle_list_.resize(L + 1);
    obstacles_[0] = lvl0;
    for (size_t l = 0; l <= L && !lvl0.empty(); l++) {
        if (l > 0) {
            for (const auto &fine : obstacles_[l - 1]) {
                std::array<size_t, 3> st{}, en{};
                for (int a = 0; a < 3; a++) {
                    st[a] = (fine.start[a] + 1) / 2;
                    en[a] = (fine.end[a] + 1) / 2;
                }
                obstacles_[l].push_back(make_box(fine.name, st, en, grid_.level(l)));
            }
        }
        IdxList merged = obstacles_[l][0].cells;
        for (size_t o = 1; o < obstacles_[l].size(); o++)
            merged = l == 0 ? merge_keep(merged, obstacles_[l][o].cells) : merge_unique(merged, obstacles_[l][o].cells);
        obstacle_list_[l] = merged;
    }

    // domain lists per level (Domain.cpp:36-252)
    inner_.resize(L + 1);
    domain_.resize(L + 1);
    boundary_.resize(L + 1);
    for (size_t l = 0; l <= L; l++) {
        const GridLevel &g = grid_.level(l);
        for (int axis = 0; axis < 3; axis++) {
            const int a1 = axis == 0 ? 1 : 0;
            const int a2 = axis == 2 ? 1 : 2;
            const int ps = 2 * axis, pe = 2 * axis + 1;
            IdxList &Ls = boundary_[l][ps], &Le = boundary_[l][pe];
            std::array<size_t, 3> cs{}, ce{};
            cs[axis] = g.cd_start[axis] - 1;
            ce[axis] = g.cd_end[axis] + 1;
            for (size_t k = g.cd_start[a2] - 1; k <= g.cd_end[a2] + 1; k++) {
                cs[a2] = ce[a2] = k;
                for (size_t j = g.cd_start[a1] - 1; j <= g.cd_end[a1] + 1; j++) {
                    cs[a1] = ce[a1] = j;
                    Ls.push_back(g.index(cs[0], cs[1], cs[2]));
                    Le.push_back(g.index(ce[0], ce[1], ce[2]));
                }
            }
        }
        const IdxList &obst = obstacle_list_[l];
        IdxList &inner = inner_[l];
        size_t cnt = 0;
        for (size_t k = g.cd_start[2]; k <= g.cd_end[2]; k++)
            for (size_t j = g.cd_start[1]; j <= g.cd_end[1]; j++)
                for (size_t i = g.cd_start[0]; i <= g.cd_end[0]; i++) {
                    const Idx idx = g.index(i, j, k);
                    if (cnt < obst.size() && obst[cnt] == idx) cnt++;
                    else inner.push_back(idx);
                }
        const size_t box = (g.cd_end[0] - g.cd_start[0] + 1) * (g.cd_end[1] - g.cd_start[1] + 1) *
                           (g.cd_end[2] - g.cd_start[2] + 1);
        if (inner.size() + obst.size() != box)
            throw config_error("obstacles overlap on multigrid level " + std::to_string(l) +
                               "; the reference list construction (src/domain/Domain.cpp:50-54, 191-203) is undefined there");
        IdxList all = boundary_[l][0];
        for (int p = 1; p < 6; p++) all = merge_unique(all, boundary_[l][p]);
        domain_[l] = merge_keep(inner, all);
    }
}

bool Geometry::has_boundary(int field_type) const {
    if (domain_bc_[field_type].present) return true;
    for (const auto &t : obstacle_bc_)
        if (t[field_type].present) return true;
    return false;
}

std::vector<BcAssign> Geometry::boundary_program(size_t level, int ft) const {
    std::vector<BcAssign> ops;
    const GridLevel &g = grid_.level(level);
    const Idx Nx = (Idx) g.N[0], Nxy = (Idx) (g.N[0] * g.N[1]);
    auto ref_of = [&](int p) -> Idx { return p >= FRONT ? Nxy : (p >= BOTTOM ? Nx : 1); };
    // obstacles in id order (ObstacleBoundary.cpp:26-213)
    for (size_t id = 0; id < obstacle_count(); id++) {
        const FieldBc &bd = obstacle_bc_[id][ft];
        if (!bd.present) continue;
        const ObstacleBox &ob = obstacles_[level][id];
        for (int p = 0; p < 6; p++) {
            const IdxList &cells = ob.patch[p];
            if (cells.empty()) continue;
            const Idx ref = (p == FRONT || p == BOTTOM || p == LEFT) ? -ref_of(p) : ref_of(p);
            if (bd.bc[p] == BC_DIRICHLET) {
                double v = bd.value[p];
                if (level > 0) v = 0;
                for (Idx t : cells) ops.push_back({t, t + ref, v * 2, -1, 0});
            } else if (bd.bc[p] == BC_NEUMANN) {
                double v = bd.value[p];
                if (level > 0) v = 0;
                v *= (p >= FRONT) ? g.spacing[2] : (p >= BOTTOM ? g.spacing[1] : g.spacing[0]);
                for (Idx t : cells) ops.push_back({t, t + ref, -v, 1, 0});
            }
            // periodic obstacle boundaries are rejected by the reference at run time
            // (ObstacleBoundary.cpp:196-200) and apply nothing
        }
    }
    // domain patches LEFT..BACK (DomainBoundary.cpp:193-238)
    const FieldBc &bd = domain_bc_[ft];
    if (bd.present) {
        for (int p = 0; p < 6; p++) {
            const IdxList &cells = boundary_[level][p];
            if (cells.empty()) continue;
            const bool neg = (p == BACK || p == TOP || p == RIGHT);
            if (bd.bc[p] == BC_DIRICHLET) {
                const double v = level == 0 ? bd.value[p] : 0;
                const Idx ref = neg ? -ref_of(p) : ref_of(p);
                for (Idx t : cells) ops.push_back({t, t + ref, v * 2, -1, 0});
            } else if (bd.bc[p] == BC_NEUMANN) {
                double v = level == 0 ? bd.value[p] : 0;
                // the reference scales LEFT/RIGHT values by dz (DomainBoundary.cpp:118-121)
                v *= (p >= FRONT) ? g.spacing[2] : (p >= BOTTOM ? g.spacing[1] : g.spacing[2]);
                const Idx ref = neg ? -ref_of(p) : ref_of(p);
                for (Idx t : cells) ops.push_back({t, t + ref, v, 1, 0});
            } else if (bd.bc[p] == BC_PERIODIC) {
                const Idx r = p >= FRONT ? Nxy * (Idx) g.n[2] : (p >= BOTTOM ? Nx * (Idx) g.n[1] : (Idx) g.n[0]);
                const Idx ref = neg ? -r : r;
                for (Idx t : cells) ops.push_back({t, t + ref, 0.0, 1, 0});
            }
        }
    }
    return ops;
}

bool Geometry::blocked(const std::array<size_t, 3> &from, const std::array<size_t, 3> &to) const {
    if (obstacles_.empty()) return false;
    for (const auto &o : obstacles_[0])
        if (o.intersects(from, to)) return true;
    return false;
}

}  // namespace artss
