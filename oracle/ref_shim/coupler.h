// Single-rank stand-in for the reference's core::Coupler (model/core/coupler.h)
// with just the members that model/modules/dynamics_rk.h calls
// (TEST INFRASTRUCTURE ONLY; see main_header.h in this directory).
//
// Semantics kept from the reference:
//   * options: typed key/value store; a missing key or a wrong type throws
//     (Options.h:122-148 aborts);
//   * DataManager: named arrays registered and fetched by type and rank
//     (DataManager.h:127-299);
//   * grid getters, tracer registry (coupler.h:234-471);
//   * halo exchanges at one rank, where every neighbour is this rank
//     (coupler.h:201-211): periodic x then y wraps (coupler.h:785-1165).
//     Indices wrap modulo n, which matches the reference whenever the halo is
//     no wider than the domain and defines the case it leaves undefined;
//   * ParallelComm::send_receive at one rank: each receive buffer takes the
//     send buffer with the same tag (ParallelComm.h:85-127);
//     all_reduce at one rank returns a copy (ParallelComm.h:247-293).
#pragma once

#include "main_header.h"
#include "MultipleFields.h"

#include <any>

namespace core {

template <class T, int N>
struct SendRecvPack {
  yakl::Array<T, N, yakl::memDevice, yakl::styleC> arr;
  int them;
  int tag;
};

class ParallelComm {
 public:
  int get_size() const { return 1; }
  int get_rank_id() const { return 0; }
  void barrier() const {}
  template <class T, int N>
  void send_receive(std::vector<SendRecvPack<T, N>> receives, std::vector<SendRecvPack<T, N>> sends,
                    std::string = "") const {
    for (auto &r : receives) {
      bool found = false;
      for (auto &s : sends)
        if (s.tag == r.tag) { s.arr.deep_copy_to(r.arr); found = true; break; }
      if (!found) Kokkos::abort("send_receive: unmatched tag");
    }
  }
  template <class T, int N, int M, int S>
  yakl::Array<typename std::remove_cv<T>::type, N, M, S> all_reduce(yakl::Array<T, N, M, S> const &a, MPI_Op) const {
    return a.template copy_as<M>();
  }
  template <class T, int N, int M, int S>
  yakl::Array<typename std::remove_cv<T>::type, N, M, S> all_reduce(yakl::Array<T, N, M, S> const &a, MPI_Op,
                                                                     std::string) const {
    return a.template copy_as<M>();
  }
  template <class T>
  T all_reduce(T v, MPI_Op) const { return v; }
  template <class T>
  T all_reduce(T v, MPI_Op, std::string) const { return v; }
  // broadcast of one value at one rank: nothing moves (ParallelComm.h:184-188).
  template <class T>
  void broadcast(T &, int = 0, std::string = "") const {}
};

class DataManager {
  struct Entry {
    std::shared_ptr<void> arr;
    size_t type_hash;
    int rank;
  };
  std::map<std::string, Entry> entries;

  template <class T, int N>
  static std::shared_ptr<void> make(std::string const &name, std::vector<int> const &d) {
    return std::make_shared<yakl::Array<T, N, memDevice, styleC>>(name.c_str(), d);
  }

 public:
  template <class T>
  void register_and_allocate(std::string name, std::string, std::vector<int> dims,
                             std::vector<std::string> = {}) {
    if (entries.count(name)) Kokkos::abort(("DataManager: entry exists: " + name).c_str());
    Entry e;
    e.type_hash = typeid(T).hash_code();
    e.rank = int(dims.size());
    switch (e.rank) {
      case 1: e.arr = make<T, 1>(name, dims); break;
      case 2: e.arr = make<T, 2>(name, dims); break;
      case 3: e.arr = make<T, 3>(name, dims); break;
      case 4: e.arr = make<T, 4>(name, dims); break;
      case 5: e.arr = make<T, 5>(name, dims); break;
      default: Kokkos::abort("DataManager: unsupported rank");
    }
    entries[name] = e;
  }
  bool entry_exists(std::string name) const { return entries.count(name) > 0; }
  template <class T, int N>
  yakl::Array<T, N, memDevice, styleC> get(std::string name) const {
    typedef typename std::remove_cv<T>::type TT;
    auto it = entries.find(name);
    if (it == entries.end()) Kokkos::abort(("DataManager: no entry " + name).c_str());
    if (it->second.type_hash != typeid(TT).hash_code() || it->second.rank != N)
      Kokkos::abort(("DataManager: wrong type or rank for " + name).c_str());
    return *static_cast<yakl::Array<TT, N, memDevice, styleC> *>(it->second.arr.get());
  }
};

class Coupler {
  std::map<std::string, std::any> options;
  std::vector<std::string> tracer_names;
  struct TracerInfo { std::string desc; bool positive, adds_mass, diffuse; };
  std::vector<TracerInfo> tracer_info;
  DataManager dm;
  ParallelComm par_comm;
  int nx, ny, nz;
  real xlen, ylen, zlen;
  SArray<int, 2, 3, 3> neigh;
  std::vector<std::function<void(Coupler &, yakl::SimplePNetCDF &)>> out_write_funcs, restart_read_funcs;

 public:
  int static constexpr DIMS_COLUMN = 1;
  int static constexpr DIMS_SURFACE = 2;
  int static constexpr DIMS_3D = 3;

  Coupler(int nx_, int ny_, int nz_, real xlen_, real ylen_, real zlen_)
      : nx(nx_), ny(ny_), nz(nz_), xlen(xlen_), ylen(ylen_), zlen(zlen_) {
    neigh = 0;
  }

  int get_nx() const { return nx; }
  int get_ny() const { return ny; }
  int get_nz() const { return nz; }
  size_t get_nx_glob() const { return nx; }
  size_t get_ny_glob() const { return ny; }
  real get_xlen() const { return xlen; }
  real get_ylen() const { return ylen; }
  real get_zlen() const { return zlen; }
  real get_dx() const { return xlen / nx; }
  real get_dy() const { return ylen / ny; }
  real get_dz() const { return zlen / nz; }
  int get_px() const { return 0; }
  int get_py() const { return 0; }
  int get_nproc_x() const { return 1; }
  int get_nproc_y() const { return 1; }
  size_t get_i_beg() const { return 0; }
  size_t get_j_beg() const { return 0; }
  bool is_sim2d() const { return ny == 1; }
  bool is_mainproc() const { return true; }
  ParallelComm get_parallel_comm() const { return par_comm; }
  SArray<int, 2, 3, 3> const &get_neighbor_rankid_matrix() const { return neigh; }
  DataManager const &get_data_manager_readonly() const { return dm; }
  DataManager &get_data_manager_readwrite() { return dm; }

  template <class T>
  void set_option(std::string key, T value) { options[key] = value; }
  bool option_exists(std::string key) const { return options.count(key) > 0; }
  template <class T>
  T get_option(std::string key) const {
    auto it = options.find(key);
    if (it == options.end()) Kokkos::abort(("missing option " + key).c_str());
    const T *v = std::any_cast<T>(&it->second);
    if (!v) Kokkos::abort(("wrong option type for " + key).c_str());
    return *v;
  }
  template <class T>
  T get_option(std::string key, T val) const { return option_exists(key) ? get_option<T>(key) : val; }

  int get_num_tracers() const { return int(tracer_names.size()); }
  std::vector<std::string> get_tracer_names() const { return tracer_names; }
  int add_tracer(std::string name, std::string desc = "", bool positive = true, bool adds_mass = false, bool diffuse = true) {
    dm.register_and_allocate<real>(name, desc, {nz, ny, nx});
    tracer_names.push_back(name);
    tracer_info.push_back({desc, positive, adds_mass, diffuse});
    return int(tracer_names.size()) - 1;
  }
  void get_tracer_info(std::string name, std::string &desc, bool &found, bool &positive, bool &adds_mass, bool &diffuse) const {
    for (size_t i = 0; i < tracer_names.size(); i++)
      if (tracer_names[i] == name) {
        desc = tracer_info[i].desc; positive = tracer_info[i].positive;
        adds_mass = tracer_info[i].adds_mass; diffuse = tracer_info[i].diffuse;
        found = true;
        return;
      }
    found = false;
  }

  template <class T>
  void register_output_variable(std::string, int) {}
  void register_write_output_module(std::function<void(Coupler &, yakl::SimplePNetCDF &)> f) { out_write_funcs.push_back(f); }
  void register_overwrite_with_restart_module(std::function<void(Coupler &, yakl::SimplePNetCDF &)> f) { restart_read_funcs.push_back(f); }
  // Runs the registered restart hooks (the reference calls them from
  // overwrite_with_restart, coupler.h:669-723, after reading the file).
  void run_restart_hooks(yakl::SimplePNetCDF &nc) { for (auto &f : restart_read_funcs) f(*this, nc); }

  template <class T>
  MultiField<typename std::remove_cv<T>::type, 3> create_and_exchange_halos(MultiField<T, 3> const &fields_in, int hs) {
    typedef typename std::remove_cv<T>::type TN;
    MultiField<TN, 3> out;
    for (int f = 0; f < fields_in.get_num_fields(); f++) {
      auto in = fields_in.get_field(f);
      int n0 = in.extent(0), n1 = in.extent(1), n2 = in.extent(2);
      yakl::Array<TN, 3, memDevice, styleC> r(in.label(), n0 + 2 * hs, n1 + 2 * hs, n2 + 2 * hs);
      for (int k = 0; k < n0; k++)
        for (int j = 0; j < n1 + 2 * hs; j++)
          for (int i = 0; i < n2 + 2 * hs; i++)
            r(hs + k, j, i) = in(k, ((j - hs) % n1 + n1) % n1, ((i - hs) % n2 + n2) % n2);
      out.add_field(r);
    }
    return out;
  }

  // Periodic x then y exchange of fields that carry hs halos on every side
  // (coupler.h:785-855 at one rank): the y pass spans the x halos, so the
  // corner halos wrap in both directions.
  template <class T>
  void halo_exchange(MultiField<T, 3> &fields, int hs) const {
    for (int f = 0; f < fields.get_num_fields(); f++) {
      auto a = fields.get_field(f);
      int nzl = a.extent(0) - 2 * hs, nyl = a.extent(1) - 2 * hs, nxl = a.extent(2) - 2 * hs;
      for (int k = 0; k < nzl; k++)
        for (int j = 0; j < nyl; j++)
          for (int ii = 0; ii < hs; ii++) {
            a(hs + k, hs + j, ii) = a(hs + k, hs + j, nxl + ii);
            a(hs + k, hs + j, nxl + hs + ii) = a(hs + k, hs + j, hs + ii);
          }
      for (int k = 0; k < nzl; k++)
        for (int jj = 0; jj < hs; jj++)
          for (int i = 0; i < nxl + 2 * hs; i++) {
            a(hs + k, jj, i) = a(hs + k, nyl + jj, i);
            a(hs + k, nyl + hs + jj, i) = a(hs + k, hs + jj, i);
          }
    }
  }

  template <class T>
  void halo_exchange_x(yakl::Array<T, 4, memDevice, styleC> const &f, int hs) const {
    int np = f.extent(0), nzl = f.extent(1) - 2 * hs, nyl = f.extent(2) - 2 * hs, nxl = f.extent(3) - 2 * hs;
#pragma omp parallel for collapse(2)
    for (int v = 0; v < np; v++)
      for (int k = 0; k < nzl; k++)
        for (int j = 0; j < nyl; j++)
          for (int ii = 0; ii < hs; ii++) {
            f(v, hs + k, hs + j, ii) = f(v, hs + k, hs + j, hs + ((ii - hs) % nxl + nxl) % nxl);
            f(v, hs + k, hs + j, nxl + hs + ii) = f(v, hs + k, hs + j, hs + ii % nxl);
          }
  }

  template <class T>
  void halo_exchange_y(yakl::Array<T, 4, memDevice, styleC> const &f, int hs) const {
    int np = f.extent(0), nzl = f.extent(1) - 2 * hs, nyl = f.extent(2) - 2 * hs, nxl = f.extent(3) - 2 * hs;
#pragma omp parallel for collapse(2)
    for (int v = 0; v < np; v++)
      for (int k = 0; k < nzl; k++)
        for (int jj = 0; jj < hs; jj++)
          for (int i = 0; i < nxl; i++) {
            f(v, hs + k, jj, hs + i) = f(v, hs + k, hs + ((jj - hs) % nyl + nyl) % nyl, hs + i);
            f(v, hs + k, nyl + hs + jj, hs + i) = f(v, hs + k, hs + jj % nyl, hs + i);
          }
  }
};

}  // namespace core
