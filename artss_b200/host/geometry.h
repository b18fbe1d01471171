// Host-side geometry of one scene: multigrid level sizes, obstacles, the
// index lists ("GPU lists") and the ordered boundary assignments.
//
// Reproduces, bit for bit, what ARTSS builds in DomainData
// (src/domain/DomainData.cpp:12-56), Obstacle (src/domain/Obstacle.cpp),
// Domain (src/domain/Domain.cpp) and Multigrid (src/domain/Multigrid.cpp),
// with one C++ object per concept and no singletons.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

#include "settings.h"

namespace artss {

using Idx = int64_t;
using IdxList = std::vector<Idx>;

// DomainData equivalent
struct GridLevel {
    std::array<size_t, 3> n{};        // inner cells (nx, ny, nz)
    std::array<size_t, 3> N{};        // cells incl. ghosts (Nx, Ny, Nz)
    std::array<double, 3> spacing{};  // dx, dy, dz
    std::array<size_t, 3> cd_start{}, cd_end{};  // computational-domain inner index range
    size_t size() const { return N[0] * N[1] * N[2]; }
    Idx index(size_t i, size_t j, size_t k) const { return (Idx) (i + N[0] * j + N[0] * N[1] * k); }
};

class Grid {
 public:
    Grid(const settings::Domain &d, size_t levels);
    size_t levels() const { return levels_; }
    const GridLevel &level(size_t l) const { return lv_[l]; }
    double length_cd(int axis) const;
    std::array<double, 3> start_pd, end_pd, start_cd, end_cd, length_pd;

 private:
    size_t levels_;
    std::vector<GridLevel> lv_;
};

// One obstacle on one level.
struct ObstacleBox {
    std::string name;
    std::array<size_t, 3> start{}, end{};
    std::array<IdxList, 6> patch;       // patch cell lists, ascending
    IdxList cells;                      // all obstacle cells, ascending
    bool contains(double x, double y, double z) const;  // is_obstacle_cell on (possibly real) indices
    // line-of-sight test of Obstacle::intersection (src/domain/Obstacle.cpp:909-978)
    bool intersects(const std::array<size_t, 3> &source, const std::array<size_t, 3> &cell) const;
};

// Boundary data of one field type: per patch condition and value (BoundaryData).
struct FieldBc {
    bool present = false;
    std::array<int, 6> bc{};
    std::array<bool, 6> has_value{};
    std::array<double, 6> value{};
};
using BcTable = std::array<FieldBc, 7>;  // by field type

// One boundary assignment x[target] = sign * x[source] + value.
struct BcAssign {
    Idx target;
    Idx source;
    double value;
    int32_t sign;
    int32_t reserved;
};

class Geometry {
 public:
    explicit Geometry(const settings::Settings &s);

    const Grid &grid() const { return grid_; }
    size_t levels() const { return grid_.levels(); }
    size_t obstacle_count() const { return obstacles_.empty() ? 0 : obstacles_[0].size(); }

    const IdxList &inner(size_t l) const { return inner_[l]; }
    const IdxList &domain(size_t l) const { return domain_[l]; }
    const IdxList &boundary(size_t l, int patch) const { return boundary_[l][patch]; }
    const IdxList &obstacle_cells(size_t l) const { return obstacle_list_[l]; }
    const ObstacleBox &obstacle(size_t l, size_t id) const { return obstacles_[l][id]; }

    // ordered assignments of Multigrid::apply_boundary_condition for one
    // field type on one level
    std::vector<BcAssign> boundary_program(size_t level, int field_type) const;
    bool has_boundary(int field_type) const;

    // DomainController::is_blocked_by_obstacle on level 0
    bool blocked(const std::array<size_t, 3> &from, const std::array<size_t, 3> &to) const;

 private:
    Grid grid_;
    std::vector<std::vector<ObstacleBox>> obstacles_;  // [level][id]
    std::vector<IdxList> obstacle_list_;               // merged obstacle cells per level
    std::vector<IdxList> inner_, domain_;
    std::vector<std::array<IdxList, 6>> boundary_;
    BcTable domain_bc_{};
    std::vector<BcTable> obstacle_bc_;
};

// Merges of ARTSS src/utility/Algorithm.cpp: `merge_keep` keeps equal
// elements of both inputs (Algorithm::merge_sort), `merge_unique` emits an
// element present in both inputs once (Algorithm::merge_sort_with_duplicates).
IdxList merge_keep(const IdxList &a, const IdxList &b);
IdxList merge_unique(const IdxList &a, const IdxList &b);

}  // namespace artss
