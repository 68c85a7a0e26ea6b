// fot_problem.hpp -- the reference's host API (Problem<SOA>, Mesh, data_t and
// the loop drivers) rebuilt on libfot's C ABI (fot.h), header-only.
//
// A program written against the reference's problem.hpp keeps its calls:
//
//   Problem<false> problem({&mesh_res, &mesh_x, &mesh_q, &mesh_adt},
//                          {2, 2, 2, 2},
//                          {{4, sizeof(double)}, {2, sizeof(double)},
//                           {4, sizeof(double)}, {1, sizeof(double)}},
//                          {}, 256);
//   problem.readPointData<double>(data_res, 0);  ...
//   problem.reorder();                            // GPS ordering (SCOTCH's "g")
//   problem.partition(1.001);                     // parts of block_size cells
//   problem.reorderToPartition();
//   problem.renumberPoints();
//   problem.loopGPUHierarchical<res_calc::StepGPUHierarchical>(num);
//   problem.writePointData<double>(out);          // un-permuted
//
// Mirrors (reference file:line):
//   data_t                       data_t.hpp:10-53 (host buffer; the device copy
//                                lives in the engine's problem)
//   Mesh                         mesh.hpp:23-389 (stream reader :67-98,
//                                numCells/numPoints/numMappings, writeCellList)
//   Problem<SOA>                 problem.hpp:29-652: constructor :59-77, loop
//                                drivers :90-437, reorder :439-482, partition
//                                :484-515, reorderToPartition :517-526,
//                                renumberPoints :528-551, partition and data
//                                I/O :553-632, calcDataSize :634-651
// The loop is identified from the point / cell data parameters (each app's
// initProblem binding is unique); the UserFunc template argument of the loop
// drivers selects the executor only.  Errors throw fot::compat::Error (the
// reference calls exit() through checkCudaErrors).
#ifndef FOT_PROBLEM_HPP
#define FOT_PROBLEM_HPP

#include <cstdint>
#include <cstring>
#include <istream>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "fot.h"

#ifndef MY_SIZE
#define MY_SIZE std::uint32_t
#endif

namespace fot {
namespace compat {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc) {
  if (rc != FOT_OK) throw Error(rc, fot_last_error());
}

// Thrown for malformed inputs, like the reference's InvalidInputFile (mesh.hpp:18-21).
struct InvalidInputFile {
  std::string input_type;
  MY_SIZE mapping_ind, line;
};

constexpr MY_SIZE DEFAULT_BLOCK_SIZE = 128;

// Host buffer of `size` elements of `dim` values of `type_size` bytes.
class data_t {
  MY_SIZE size_ = 0, dim_ = 0;
  unsigned type_size_ = 0;
  std::vector<char> data_;

 public:
  data_t(MY_SIZE size, MY_SIZE dim, unsigned type_size)
      : size_(size), dim_(dim), type_size_(type_size), data_((size_t)size * dim * type_size) {}
  template <typename T> static data_t create(MY_SIZE size, MY_SIZE dim) {
    return data_t(size, dim, sizeof(T));
  }
  template <typename T = char> T &operator[](MY_SIZE i) {
    return *reinterpret_cast<T *>(data_.data() + (size_t)i * type_size_);
  }
  template <typename T = char> const T &operator[](MY_SIZE i) const {
    return *reinterpret_cast<const T *>(data_.data() + (size_t)i * type_size_);
  }
  template <typename T = char> T *begin() { return reinterpret_cast<T *>(data_.data()); }
  template <typename T = char> T *end() { return reinterpret_cast<T *>(data_.data() + data_.size()); }
  template <typename T = char> const T *cbegin() const { return reinterpret_cast<const T *>(data_.data()); }
  template <typename T = char> const T *cend() const {
    return reinterpret_cast<const T *>(data_.data() + data_.size());
  }
  MY_SIZE getSize() const { return size_; }
  MY_SIZE getDim() const { return dim_; }
  unsigned getTypeSize() const { return type_size_; }
  size_t bytes() const { return data_.size(); }
};

// data_t.hpp:104-114
template <bool SOA = false>
inline MY_SIZE index(MY_SIZE num_points, MY_SIZE node_ind, MY_SIZE Dim, MY_SIZE dim) {
  return SOA ? dim * num_points + node_ind : node_ind * Dim + dim;
}

class Mesh {
  std::vector<MY_SIZE> num_points_;

 public:
  std::vector<data_t> cell_to_node;

  // Text format of the reference (mesh.hpp:57-98): "num_points num_cells",
  // then num_cells lines of mesh_dim point ids.
  Mesh(const std::vector<std::istream *> &iis, const std::vector<MY_SIZE> &mesh_dim) {
    MY_SIZE num_cells = 0;
    for (size_t k = 0; k < iis.size(); ++k) {
      std::istream &is = *iis[k];
      if (!is) throw InvalidInputFile{"graph input", (MY_SIZE)k, 0};
      MY_SIZE np = 0, nc = 0;
      is >> np >> nc;
      if (!is || (k > 0 && nc != num_cells)) throw InvalidInputFile{"graph input", (MY_SIZE)k, 0};
      num_cells = nc;
      num_points_.push_back(np);
      cell_to_node.push_back(data_t::create<MY_SIZE>(nc, mesh_dim[k]));
      for (MY_SIZE i = 0; i < nc; ++i) {
        for (MY_SIZE j = 0; j < mesh_dim[k]; ++j) {
          MY_SIZE v = 0;
          is >> v;
          cell_to_node.back().operator[]<MY_SIZE>(i * mesh_dim[k] + j) = v;
        }
        if (!is) throw InvalidInputFile{"graph input", (MY_SIZE)k, i + 1};
      }
    }
  }
  Mesh(std::vector<MY_SIZE> num_points, std::vector<data_t> maps)
      : num_points_(std::move(num_points)), cell_to_node(std::move(maps)) {}
  MY_SIZE numCells() const { return cell_to_node.at(0).getSize(); }
  MY_SIZE numPoints(unsigned k) const { return num_points_.at(k); }
  const std::vector<MY_SIZE> numPoints() const { return num_points_; }
  unsigned numMappings() const { return (unsigned)cell_to_node.size(); }
  void writeCellList(std::ostream &os, unsigned k) const {
    os << numPoints(k) << " " << numCells() << "\n";
    const MY_SIZE d = cell_to_node[k].getDim();
    for (MY_SIZE i = 0; i < numCells(); ++i) {
      for (MY_SIZE j = 0; j < d; ++j)
        os << (j ? " " : "") << cell_to_node[k].operator[]<MY_SIZE>(i * d + j);
      os << "\n";
    }
  }
};

// Executor tags: the reference's StepSeq / StepGPUGlobal / StepGPUHierarchical
// names of each app select the executor of the loop drivers below.
#define FOT_COMPAT_APP(name)                                                   \
  namespace name {                                                             \
  struct StepGPUGlobal {};                                                     \
  struct StepGPUHierarchical {};                                               \
  }
FOT_COMPAT_APP(res_calc)
FOT_COMPAT_APP(mini_aero)
FOT_COMPAT_APP(lulesh)
FOT_COMPAT_APP(volna)
FOT_COMPAT_APP(getacc)
#undef FOT_COMPAT_APP

template <bool SOA = false> class Problem {
 public:
  Mesh mesh;
  std::vector<data_t> point_weights;
  std::vector<data_t> cell_weights;
  const MY_SIZE block_size;
  std::vector<MY_SIZE> partition_vector;
  std::vector<MY_SIZE> applied_permutation;

  Problem(const std::vector<std::istream *> &mesh_is, const std::vector<MY_SIZE> &mesh_dim,
          const std::vector<std::pair<MY_SIZE, unsigned>> &point_data_params,
          const std::vector<std::pair<MY_SIZE, unsigned>> &cell_data_params,
          MY_SIZE block_size_ = DEFAULT_BLOCK_SIZE)
      : mesh(mesh_is, mesh_dim), block_size(block_size_) {
    loop_ = identify(mesh_dim, point_data_params, cell_data_params);
    for (unsigned k = 0; k < mesh.numMappings(); ++k)
      point_weights.emplace_back(mesh.numPoints(k), point_data_params[k].first,
                                 point_data_params[k].second);
    for (const auto &c : cell_data_params)
      cell_weights.emplace_back(mesh.numCells(), c.first, c.second);
    std::vector<const uint32_t *> maps;
    for (auto &m : mesh.cell_to_node) maps.push_back(m.template cbegin<uint32_t>());
    const std::vector<MY_SIZE> np = mesh.numPoints();
    check(fot_problem_create(loop_, SOA ? FOT_SOA : FOT_AOS, mesh.numCells(), np.data(),
                             maps.data(), &h_));
  }
  ~Problem() {
    if (plan_) fot_plan_destroy(plan_);
    if (h_) fot_problem_destroy(h_);
  }
  Problem(const Problem &) = delete;
  Problem &operator=(const Problem &) = delete;

  int loopId() const { return loop_; }

  // ---- loop drivers (problem.hpp:90-437) ----------------------------------
  template <class UserFunc> void loopGPUCellCentred(MY_SIZE num) {
    run(FOT_EXEC_ATOMIC, num);
  }
  template <class UserFunc, unsigned SharedMemoryMultiplier = 0>
  void loopGPUHierarchical(MY_SIZE num) {
    run(FOT_EXEC_HIER, num);
  }

  // ---- orderings (problem.hpp:439-551) -------------------------------------
  template <bool SameMapping = false> void reorder(int order = FOT_ORDER_GPS) {
    push();
    check(fot_reorder(h_, order, 1));
    pull(true);
  }
  // METIS k-way with load-balance tolerance (problem.hpp:484-499): recursive
  // graph bisection on the GPU into ceil(numCells / block_size) parts, no
  // part above tolerance x the mean (+1 cell)
  void partition(float tolerance) {
    push();
    check(fot_partition_tol(h_, block_size, tolerance, FOT_PARTITION_BISECT));
    pull(true);
  }
  // METIS coarse parts of block_size x num_blocks_in_coarse cells refined by
  // the heuristic growth (problem.hpp:501-515): the bisection is already
  // hierarchical -- its first rounds cut the coarse parts -- so the fine
  // parts come from the same call
  void partitionOurs(float tolerance, MY_SIZE /*num_blocks_in_coarse*/) { partition(tolerance); }
  void reorderToPartition() {
    push();
    check(fot_reorder_to_partition(h_));
    pull(true);
  }
  void renumberPoints() {
    push();
    check(fot_renumber_points(h_));
    pull(true);
  }

  // ---- data I/O (problem.hpp:553-632) --------------------------------------
  template <class DataType> void readPointData(std::istream &is, unsigned k) {
    if (!is) throw InvalidInputFile{"point data input", k, 0};
    data_t &d = point_weights.at(k);
    for (MY_SIZE i = 0; i < mesh.numPoints(k); ++i) {
      for (MY_SIZE j = 0; j < d.getDim(); ++j)
        is >> d.template operator[]<DataType>(index<SOA>(d.getSize(), i, d.getDim(), j));
      if (!is && !is.eof()) throw InvalidInputFile{"point data input", k, i};
    }
    dirty_ = true;
  }
  template <class DataType> void readCellData(std::istream &is, unsigned k) {
    if (!is) throw InvalidInputFile{"cell data input", k, 0};
    data_t &d = cell_weights.at(k);
    for (MY_SIZE i = 0; i < mesh.numCells(); ++i) {
      for (MY_SIZE j = 0; j < d.getDim(); ++j)
        is >> d.template operator[]<DataType>(j * d.getSize() + i);
      if (!is) throw InvalidInputFile{"cell data input", k, i};
    }
    dirty_ = true;
  }
  template <class DataType> void writePointData(std::ostream &os) const {
    const MY_SIZE n = mesh.numPoints(0), dim = point_weights[0].getDim();
    for (MY_SIZE i = 0; i < n; ++i) {
      for (MY_SIZE j = 0; j < dim; ++j) {
        const MY_SIZE p = applied_permutation.empty() ? i : applied_permutation[i];
        os << (j ? " " : "") << point_weights[0].template operator[]<DataType>(index<SOA>(n, p, dim, j));
      }
      os << "\n";
    }
  }
  void writePartition(std::ostream &os) const {
    os << block_size << "\n";
    for (MY_SIZE p : partition_vector) os << p << "\n";
  }
  void readPartition(std::istream &is) {
    MY_SIZE bs = 0;
    is >> bs;
    if (!is) throw InvalidInputFile{"partition input", 0, 1};
    partition_vector.resize(mesh.numCells());
    for (MY_SIZE i = 0; i < mesh.numCells(); ++i) {
      is >> partition_vector[i];
      if (!is) throw InvalidInputFile{"partition input", 0, i + 1};
    }
    check(fot_set_partition(h_, partition_vector.data()));
  }

  // problem.hpp:634-651 (counts every mapping, as the reference does)
  double calcDataSize() const {
    double r = 0;
    for (unsigned k = 0; k < mesh.numMappings(); ++k)
      r += point_weights[k].bytes() + mesh.cell_to_node[k].bytes();
    for (const auto &c : cell_weights) r += c.bytes();
    return r + point_weights[0].bytes();
  }

 private:
  int loop_ = -1;
  fot_problem *h_ = nullptr;
  fot_plan *plan_ = nullptr;
  int plan_exec_ = -1;
  bool dirty_ = true;

  static int identify(const std::vector<MY_SIZE> &mesh_dim,
                      const std::vector<std::pair<MY_SIZE, unsigned>> &pp,
                      const std::vector<std::pair<MY_SIZE, unsigned>> &cp) {
    for (int loop = 0; loop < FOT_NUM_LOOPS; ++loop) {
      fot_loop_info info;
      check(fot_loop_describe(loop, &info));
      if (info.n_mappings != mesh_dim.size() || info.n_point_sets != pp.size() ||
          info.n_cell_sets != cp.size())
        continue;
      bool ok = true;
      for (size_t k = 0; k < pp.size(); ++k)
        ok = ok && info.mesh_dim[k] == mesh_dim[k] && info.point_dim[k] == pp[k].first &&
             info.point_type_size[k] == pp[k].second;
      for (size_t j = 0; j < cp.size(); ++j)
        ok = ok && info.cell_dim[j] == cp[j].first && info.cell_type_size[j] == cp[j].second;
      if (ok) return loop;
    }
    throw Error(FOT_ERR_ARG, "the data parameters match none of the engine's loops");
  }

  // The host mirrors keep the cell order of the last explicit ordering call
  // (as the reference's Problem does); a hierarchical plan build puts the
  // engine's cells in plan order, so host position host_pos_[i] holds the
  // engine's cell i.
  std::vector<MY_SIZE> host_pos_;
  std::vector<MY_SIZE> user_order_;

  void refresh_host_pos() {
    const MY_SIZE n = mesh.numCells();
    std::vector<MY_SIZE> dev(n), inv(n);
    check(fot_get_cell_order(h_, dev.data()));
    if (user_order_.size() != n) user_order_ = dev;
    for (MY_SIZE i = 0; i < n; ++i) inv[user_order_[i]] = i;
    host_pos_.resize(n);
    for (MY_SIZE i = 0; i < n; ++i) host_pos_[i] = inv[dev[i]];
  }
  // host -> device: the datasets (the reference's initDeviceMemory)
  void push() {
    if (!dirty_) return;
    refresh_host_pos();
    for (unsigned k = 0; k < point_weights.size(); ++k)
      check(fot_set_point_data(h_, k, point_weights[k].begin(), point_weights[k].bytes()));
    for (unsigned j = 0; j < cell_weights.size(); ++j) {
      const data_t &c = cell_weights[j];
      std::vector<char> buf(c.bytes());
      const MY_SIZE n = c.getSize(), ts = c.getTypeSize();
      for (MY_SIZE d = 0; d < c.getDim(); ++d)
        for (MY_SIZE i = 0; i < n; ++i)
          std::memcpy(&buf[((size_t)d * n + i) * ts], c.cbegin() + ((size_t)d * n + host_pos_[i]) * ts, ts);
      check(fot_set_cell_data(h_, j, buf.data(), buf.size()));
    }
    dirty_ = false;
  }
  // device -> host: the datasets
  void pull_data() {
    refresh_host_pos();
    for (unsigned k = 0; k < point_weights.size(); ++k)
      check(fot_get_point_data(h_, k, point_weights[k].begin(), point_weights[k].bytes()));
    for (unsigned j = 0; j < cell_weights.size(); ++j) {
      data_t &c = cell_weights[j];
      std::vector<char> buf(c.bytes());
      check(fot_get_cell_data(h_, j, buf.data(), buf.size()));
      const MY_SIZE n = c.getSize(), ts = c.getTypeSize();
      for (MY_SIZE d = 0; d < c.getDim(); ++d)
        for (MY_SIZE i = 0; i < n; ++i)
          std::memcpy(c.begin() + ((size_t)d * n + host_pos_[i]) * ts, &buf[((size_t)d * n + i) * ts], ts);
    }
  }
  // after an explicit ordering call: the engine's order becomes the host's
  void pull(bool topology) {
    if (topology) {
      user_order_.clear();  // adopt the engine's current cell order
      refresh_host_pos();
      for (unsigned k = 0; k < mesh.numMappings(); ++k)
        check(fot_get_mapping(h_, k, mesh.cell_to_node[k].template begin<uint32_t>()));
      applied_permutation.resize(mesh.numPoints(0));
      check(fot_get_point_permutation(h_, 0, applied_permutation.data()));
      partition_vector.resize(mesh.numCells());
      if (fot_get_partition(h_, partition_vector.data()) != FOT_OK) partition_vector.clear();
      if (plan_) {
        fot_plan_destroy(plan_);
        plan_ = nullptr;
      }
    }
    pull_data();
  }
  void run(int exec, MY_SIZE num) {
    push();
    if (!plan_ || plan_exec_ != exec) {
      if (plan_) fot_plan_destroy(plan_);
      plan_ = nullptr;
      fot_plan_desc desc{exec, exec == FOT_EXEC_ATOMIC ? 256u : block_size,
                         partition_vector.size() == mesh.numCells() ? FOT_PLAN_USE_PARTITION : 0u, 0};
      check(fot_plan_build(h_, &desc, &plan_));
      plan_exec_ = exec;
    }
    check(fot_run(h_, plan_, num, nullptr));
    check(fot_sync(h_, nullptr));
    pull_data();
  }
};

} // namespace compat
} // namespace fot

#endif // FOT_PROBLEM_HPP
