// Python extension ``boltzmann_b200.boltzmann``: the classes of the reference's pyo3 module
// (djbarker/boltzmann src/lib.rs:22-411) -- Omega, Simulation, Fluid, Scalar, Cells -- with the
// host-side semantics of its Simulation (src/simulation.rs), on top of the C ABI in
// include/lbm_cuda.h. Nothing here touches CUDA directly.
//
// Host arrays are page-locked mirrors owned by the simulation state; Python sees them as
// zero-copy numpy views that keep the state alive (src/lib.rs:58-70, 94-105, 136-160).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <array>
#include <charconv>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "lbm_closure.h"
#include "lbm_cuda.h"

namespace py = pybind11;

namespace {

// Mirrors pyo3's PanicException: the reference reports misuse by panicking (src/simulation.rs
// 279-281, 315-319; src/opencl.rs:30; src/lib.rs:195, 315).
struct Panic : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check(int rc) {
  if (rc != LBM_OK) throw Panic(lbm_last_error());
}

template <class T>
struct Pinned {
  T* p = nullptr;
  size_t n = 0;
  Pinned() = default;
  Pinned(size_t count, T fill) : n(count) {
    p = static_cast<T*>(lbm_host_alloc(std::max<size_t>(count, 1) * sizeof(T)));
    if (p == nullptr) throw Panic(std::string("host allocation failed: ") + lbm_last_error());
    std::fill(p, p + count, fill);
  }
  Pinned(const Pinned&) = delete;
  Pinned& operator=(const Pinned&) = delete;
  Pinned(Pinned&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  Pinned& operator=(Pinned&& o) noexcept {
    std::swap(p, o.p);
    std::swap(n, o.n);
    return *this;
  }
  ~Pinned() { lbm_host_free(p); }
};

struct Omega {
  int kind = LBM_BGK;  // LBM_BGK or LBM_TRT
  float pos = 0, neg = 0;
};

std::string fmt_f32(float v) {
  char buf[64];
  auto r = std::to_chars(buf, buf + sizeof buf, v);
  return std::string(buf, r.ptr);
}

std::string omega_repr(const Omega& o) {
  if (o.kind == LBM_BGK) return "Omega.BGK(" + fmt_f32(o.pos) + ")";
  return "Omega.TRT(" + fmt_f32(o.pos) + ", " + fmt_f32(o.neg) + ")";
}

struct TracerState {
  int index = -1;  // index in the C ABI simulation
  int q = 0;
  Omega omega;
  Pinned<float> val;
  bool on_device = false;
};

struct Coupling {
  std::string tracer;
  float alpha = 0, c0 = 0;
  std::vector<float> g;
};

// The host model: src/simulation.rs:131-140 plus the C ABI handle.
struct SimState {
  lbm_sim* h = nullptr;
  std::vector<int64_t> counts;
  int dim = 0, q = 0, storage = LBM_STORAGE_F32;
  Omega omega;
  int64_t n = 0;
  Pinned<int32_t> flags;
  Pinned<float> rho, vel;
  std::map<std::string, TracerState> tracers;
  std::vector<std::string> tracer_order;  // C ABI index order
  std::optional<std::vector<float>> gravity;
  std::vector<Coupling> couplings;
  uint64_t iteration = 0;
  bool acc_allocated = false;
  std::recursive_mutex mu;

  ~SimState() {
    if (h) lbm_destroy(h);
  }

  int64_t fluid_bytes() const {
    // src/fields.rs:131-137: f + rho + vel (+ acc) host elements, as f32.
    int64_t acc = acc_allocated ? n * dim : 0;
    return 4 * (n * q + n + n * dim + acc);
  }
  int64_t cells_bytes() const { return 4 * n; }  // src/simulation.rs:55-59
  int64_t tracer_bytes(const TracerState& t) const { return 4 * (n * t.q + n); }

  // Simulation::finalize (src/simulation.rs:254-275): every host array to the device.
  void upload_all() {
    check(lbm_upload_flags(h, flags.p));
    check(lbm_upload_fluid(h, rho.p, vel.p));
    for (auto& name : tracer_order) {
      TracerState& t = tracers.at(name);
      check(lbm_upload_tracer(h, t.index, t.val.p));
      t.on_device = true;
    }
  }

  // Simulation::iterate (src/simulation.rs:278-446). Makes no Python API call, so callers run it
  // with the GIL released.
  void iterate(int64_t iters) {
    if (iters % 2 != 0) throw Panic("iters must be even");
    prepare();
    check(lbm_iterate(h, iters));
    read_back();
    iteration += (uint64_t)iters;
  }

  // The device-side part of the first call (upload + equilibrate), late tracers, and the
  // acceleration flag: everything iterate() does before stepping.
  void prepare() {
    if (iteration == 0) {
      upload_all();
      check(lbm_equilibrate(h));
    }
    // A tracer added after the first call: give it its host values and equilibrium.
    for (auto& name : tracer_order) {
      TracerState& t = tracers.at(name);
      if (!t.on_device) {
        check(lbm_upload_tracer(h, t.index, t.val.p));
        check(lbm_equilibrate_tracer(h, t.index));
        t.on_device = true;
      }
    }
    if (gravity || !couplings.empty()) acc_allocated = true;  // src/simulation.rs:288-295
  }

  // src/fields.rs:97-104, 177-183: device fields into the host mirrors.
  void read_back() {
    check(lbm_download_fluid(h, rho.p, vel.p));
    for (auto& name : tracer_order) {
      TracerState& t = tracers.at(name);
      check(lbm_download_tracer(h, t.index, t.val.p));
    }
  }
};

using StatePtr = std::shared_ptr<SimState>;

// Zero-copy numpy view of a mirror, keeping the state alive.
template <class T>
py::array view(const StatePtr& st, T* data, std::vector<py::ssize_t> shape) {
  auto* keep = new StatePtr(st);
  py::capsule owner(keep, [](void* p) { delete static_cast<StatePtr*>(p); });
  return py::array_t<T>(shape, data, owner);
}

std::vector<py::ssize_t> shape_of(const SimState& s, std::optional<int> extra = std::nullopt) {
  std::vector<py::ssize_t> sh(s.counts.begin(), s.counts.end());
  if (extra) sh.push_back(*extra);
  return sh;
}

int parse_storage(const std::string& s) {
  if (s == "f32" || s == "float32") return LBM_STORAGE_F32;
  if (s == "f16" || s == "float16") return LBM_STORAGE_F16;
  if (s == "bf16" || s == "bfloat16") return LBM_STORAGE_BF16;
  if (s == "f64" || s == "float64") return LBM_STORAGE_F64;
  throw py::value_error("storage must be one of 'f32', 'f16', 'bf16', 'f64'");
}

const char* storage_name(int s) {
  switch (s) {
    case LBM_STORAGE_F16: return "f16";
    case LBM_STORAGE_BF16: return "bf16";
    case LBM_STORAGE_F64: return "f64";
    default: return "f32";
  }
}

// src/opencl.rs:25-33: only "cpu" and "gpu" (any case) are device strings. Both run on the CUDA
// device here; there is no CPU fallback.
void check_device(const std::string& dev) {
  std::string u = dev;
  std::transform(u.begin(), u.end(), u.begin(), ::toupper);
  if (u != "CPU" && u != "GPU") throw Panic("Invalid device type. Expected either 'cpu' or 'gpu'.");
}

StatePtr make_state(const std::vector<int64_t>& counts, const Omega& omega, int q, int storage) {
  auto st = std::make_shared<SimState>();
  st->counts = counts;
  st->dim = (int)counts.size();
  st->q = q;
  st->storage = storage;
  st->omega = omega;
  st->n = 1;
  for (int64_t c : counts) st->n *= c;
  check(lbm_create(st->dim, counts.data(), q, omega.kind, omega.pos, omega.neg, storage, &st->h));
  st->flags = Pinned<int32_t>((size_t)st->n, 0);
  st->rho = Pinned<float>((size_t)st->n, 1.0f);
  st->vel = Pinned<float>((size_t)(st->n * st->dim), 0.0f);
  return st;
}

int default_q(int dim, bool tracer) {
  switch (dim) {
    case 1: return 3;
    case 2: return tracer ? 5 : 9;
    case 3: return tracer ? 7 : 27;
  }
  throw Panic("Invalid number of dimensions. Expected either 1, 2 or 3.");
}

std::vector<float> as_floats(py::handle obj) {
  auto a = py::array_t<float, py::array::c_style | py::array::forcecast>::ensure(obj);
  if (!a) throw py::type_error("expected a 1-D float32 array");
  return std::vector<float>(a.data(), a.data() + a.size());
}

struct Fluid {
  StatePtr st;
};
struct Cells {
  StatePtr st;
};
struct Scalar {
  StatePtr st;
  std::string name;
};

struct Simulation {
  StatePtr st;

  TracerState& tracer(const std::string& name) {
    auto it = st->tracers.find(name);
    if (it == st->tracers.end()) throw Panic("No tracers configured");
    return it->second;
  }

  Scalar add_tracer(const std::string& name, const Omega& omega, std::optional<int> q) {
    std::lock_guard<std::recursive_mutex> lock(st->mu);
    if (st->tracers.find(name) == st->tracers.end()) {
      const int tq = q ? *q : default_q(st->dim, true);
      TracerState t;
      t.q = tq;
      t.omega = omega;
      check(lbm_add_tracer(st->h, tq, omega.kind, omega.pos, omega.neg, &t.index));
      t.val = Pinned<float>((size_t)st->n, 0.0f);
      st->tracers.emplace(name, std::move(t));
      st->tracer_order.push_back(name);
    }
    return Scalar{st, name};
  }

  void set_gravity(py::handle g) {
    std::lock_guard<std::recursive_mutex> lock(st->mu);
    std::vector<float> v = as_floats(g);
    if ((int)v.size() < st->dim) throw py::value_error("gravity needs one entry per dimension");
    check(lbm_set_gravity(st->h, v.data()));
    st->gravity = v;
  }

  void add_boussinesq_coupling(const Scalar& tracer, float alpha, float c0, py::handle g) {
    std::lock_guard<std::recursive_mutex> lock(st->mu);
    std::vector<float> v = as_floats(g);
    if ((int)v.size() < st->dim) throw py::value_error("gravity needs one entry per dimension");
    auto it = st->tracers.find(tracer.name);
    if (it == st->tracers.end()) throw Panic("assertion failed: self.tracers.contains_key(tracer)");
    check(lbm_add_coupling(st->h, it->second.index, alpha, c0, v.data()));
    st->couplings.push_back(Coupling{tracer.name, alpha, c0, v});
  }

  // The GIL is released for the whole call (the reference holds it); the state mutex is taken
  // after releasing it, so no thread ever waits for the GIL while holding the mutex.
  void iterate(int64_t iters) {
    py::gil_scoped_release nogil;
    std::lock_guard<std::recursive_mutex> lock(st->mu);
    st->iterate(iters);
  }
};

// Populations in the checkpoint layout [*counts, q] (read back from the device).
py::array read_populations(const StatePtr& st, std::optional<std::string> tracer) {
  int q = st->q;
  int index = -1;
  if (tracer) {
    TracerState& t = st->tracers.at(*tracer);
    q = t.q;
    index = t.index;
  }
  py::array_t<float> out(shape_of(*st, q));
  {
    py::gil_scoped_release nogil;
    std::lock_guard<std::recursive_mutex> lock(st->mu);
    if (index < 0)
      check(lbm_download_f(st->h, out.mutable_data()));
    else
      check(lbm_download_g(st->h, index, out.mutable_data()));
  }
  return out;
}

}  // namespace

PYBIND11_MODULE(boltzmann, m) {
  m.doc() = "CUDA (sm_100a) lattice-Boltzmann backend with the Python API of djbarker/boltzmann.";
  py::register_exception<Panic>(m, "PanicException", PyExc_BaseException);

  py::class_<Omega>(m, "Omega", "Collision operator parameters (src/lib.rs:22-46).")
      .def_static(
          "BGK", [](float omega) { return Omega{LBM_BGK, omega, 0.0f}; }, py::arg("omega"))
      .def_static(
          "TRT",
          [](float omega_pos, float omega_neg) { return Omega{LBM_TRT, omega_pos, omega_neg}; },
          py::arg("omega_pos"), py::arg("omega_neg"))
      .def_property_readonly("_0", [](const Omega& o) { return o.pos; })
      .def_property_readonly("_1", [](const Omega& o) -> py::object {
        if (o.kind == LBM_TRT) return py::float_(o.neg);
        throw py::attribute_error("Omega.BGK has a single field");
      })
      .def_property_readonly("kind",
                             [](const Omega& o) { return o.kind == LBM_BGK ? "BGK" : "TRT"; })
      .def("__repr__", &omega_repr)
      .def("__eq__", [](const Omega& a, const Omega& b) {
        return a.kind == b.kind && a.pos == b.pos && (a.kind == LBM_BGK || a.neg == b.neg);
      });

  py::class_<Fluid>(m, "Fluid", "The fluid density and velocity fields (src/lib.rs:48-79).")
      .def_property_readonly("rho",
                             [](const Fluid& f) { return view(f.st, f.st->rho.p, shape_of(*f.st)); })
      .def_property_readonly(
          "vel", [](const Fluid& f) { return view(f.st, f.st->vel.p, shape_of(*f.st, f.st->dim)); })
      .def_property_readonly("size_bytes", [](const Fluid& f) { return f.st->fluid_bytes(); });

  py::class_<Scalar>(m, "Scalar", "A tracer (scalar) field (src/lib.rs:81-120).")
      .def_property_readonly("val",
                             [](const Scalar& s) {
                               auto it = s.st->tracers.find(s.name);
                               if (it == s.st->tracers.end()) throw Panic("No tracers configured");
                               return view(s.st, it->second.val.p, shape_of(*s.st));
                             })
      .def_property_readonly("size_bytes", [](const Scalar& s) {
        auto it = s.st->tracers.find(s.name);
        if (it == s.st->tracers.end())
          throw Panic("called `Option::unwrap()` on a `None` value");
        return s.st->tracer_bytes(it->second);
      });

  py::class_<Cells>(m, "Cells", "Cell flags and domain size (src/lib.rs:122-169).")
      .def_property_readonly(
          "flags", [](const Cells& c) { return view(c.st, c.st->flags.p, shape_of(*c.st)); })
      .def_property_readonly("size_bytes", [](const Cells& c) { return c.st->cells_bytes(); })
      .def_property_readonly("counts",
                             [](const Cells& c) {
                               py::array_t<uint64_t> a((py::ssize_t)c.st->counts.size());
                               for (size_t k = 0; k < c.st->counts.size(); ++k)
                                 a.mutable_data()[k] = (uint64_t)c.st->counts[k];
                               return a;
                             })
      .def_property_readonly("count", [](const Cells& c) { return (uint64_t)c.st->n; });

  py::class_<Simulation>(m, "Simulation",
                         "Domain, fluid and tracers of one lattice-Boltzmann simulation "
                         "(src/lib.rs:171-399).")
      .def(py::init([](const std::string& dev, const std::vector<int64_t>& counts,
                       const Omega& omega, std::optional<int> q, const std::string& storage,
                       std::optional<std::string> tracer_storage) {
             check_device(dev);
             const int qq = q ? *q : default_q((int)counts.size(), false);
             Simulation sim{make_state(counts, omega, qq, parse_storage(storage))};
             // Tracer populations: float by default, or the fluid's own 16-bit kind.
             if (tracer_storage)
               check(lbm_set_tracer_storage(sim.st->h, parse_storage(*tracer_storage)));
             return sim;
           }),
           py::arg("dev"), py::arg("counts"), py::arg("omega"), py::arg("q") = py::none(),
           py::arg("storage") = "f32", py::arg("tracer_storage") = py::none())
      .def_property_readonly("device_info",
                             [](const Simulation& s) {
                               char buf[256] = {0};
                               check(lbm_device_info(s.st->h, buf, sizeof buf));
                               return std::string(buf);
                             })
      .def_property_readonly("size_bytes",
                             [](const Simulation& s) {
                               int64_t b = s.st->fluid_bytes() + s.st->cells_bytes();
                               for (auto& kv : s.st->tracers) b += s.st->tracer_bytes(kv.second);
                               return b;
                             })
      .def_property_readonly("iteration", [](const Simulation& s) { return s.st->iteration; })
      .def_property_readonly("storage",
                             [](const Simulation& s) { return storage_name(s.st->storage); })
      .def("iterate", &Simulation::iterate, py::arg("iters"))
      .def("set_gravity", &Simulation::set_gravity, py::arg("gravity"))
      .def("add_boussinesq_coupling", &Simulation::add_boussinesq_coupling, py::arg("tracer"),
           py::arg("alpha"), py::arg("c0"), py::arg("g"))
      .def("add_tracer", &Simulation::add_tracer, py::arg("name"), py::arg("omega"),
           py::arg("q") = py::none())
      .def("get_tracer",
           [](const Simulation& s, const std::string& name) { return Scalar{s.st, name}; },
           py::arg("name"))
      .def_property_readonly("cells", [](const Simulation& s) { return Cells{s.st}; })
      .def_property_readonly("fluid", [](const Simulation& s) { return Fluid{s.st}; })
      .def(
          "write_checkpoint",
          [](Simulation& s, const std::string& path) {
            py::module_::import("boltzmann_b200.checkpoint").attr("write_checkpoint")(
                py::cast(s), path);
          },
          py::arg("path"))
      .def_static(
          "load_checkpoint",
          [](const std::string& dev, const std::string& path) {
            check_device(dev);
            return py::module_::import("boltzmann_b200.checkpoint").attr("load_checkpoint")(path);
          },
          py::arg("dev"), py::arg("path"))
      // -- used by boltzmann_b200.checkpoint and the tests (not part of the reference API) --
      .def("_populations", [](const Simulation& s) { return read_populations(s.st, std::nullopt); })
      .def("_tracer_populations",
           [](const Simulation& s, const std::string& name) { return read_populations(s.st, name); })
      .def("_tracer_names", [](const Simulation& s) { return s.st->tracer_order; })
      .def("_tracer_q", [](const Simulation& s, const std::string& n) { return s.st->tracers.at(n).q; })
      .def("_tracer_omega",
           [](const Simulation& s, const std::string& n) { return s.st->tracers.at(n).omega; })
      .def_property_readonly("_q", [](const Simulation& s) { return s.st->q; })
      .def_property_readonly("_omega", [](const Simulation& s) { return s.st->omega; })
      .def_property_readonly("_gravity", [](const Simulation& s) { return s.st->gravity; })
      .def_property_readonly("_acc_allocated",
                             [](const Simulation& s) { return s.st->acc_allocated; })
      .def("_couplings",
           [](const Simulation& s) {
             py::list out;
             for (const Coupling& c : s.st->couplings)
               out.append(py::make_tuple(c.tracer, c.alpha, c.c0, c.g));
             return out;
           })
      .def("_restore",
           [](Simulation& s, py::array_t<float, py::array::c_style | py::array::forcecast> f,
              py::dict tracer_g, uint64_t iteration, bool acc_allocated) {
             // Load path (src/simulation.rs:464-479): host mirrors are already filled; upload
             // everything and the populations, without equilibrating.
             std::lock_guard<std::recursive_mutex> lock(s.st->mu);
             SimState& st = *s.st;
             if ((int64_t)f.size() != st.n * st.q) throw py::value_error("f has the wrong size");
             st.upload_all();
             check(lbm_upload_f(st.h, f.data()));
             for (auto item : tracer_g) {
               const std::string name = py::cast<std::string>(item.first);
               TracerState& t = st.tracers.at(name);
               auto g = py::array_t<float, py::array::c_style | py::array::forcecast>::ensure(
                   item.second);
               if ((int64_t)g.size() != st.n * t.q) throw py::value_error("g has the wrong size");
               check(lbm_upload_g(st.h, t.index, g.data()));
             }
             st.iteration = iteration;
             st.acc_allocated = acc_allocated;
           })
      .def("_conservation",
           [](const Simulation& s) {
             std::vector<double> out(1 + s.st->dim + s.st->tracers.size());
             check(lbm_conservation(s.st->h, out.data(), (int)out.size()));
             return out;
           })
      .def("_nonfinite",
           [](const Simulation& s) {
             int flag = 0;
             check(lbm_nonfinite(s.st->h, &flag));
             return flag != 0;
           })
      .def("_fluid_f64",
           [](const Simulation& s) {
             const SimState& st = *s.st;
             py::array_t<double> rho(shape_of(st)), vel(shape_of(st, st.dim));
             check(lbm_download_fluid_f64(st.h, rho.mutable_data(), vel.mutable_data()));
             return py::make_tuple(rho, vel);
           })
      .def("_iterate_device",
           [](Simulation& s, int64_t iters) {
             // Steps only, without the read-back of iterate() (device-side drivers and timing);
             // _read_back() refreshes the host mirrors.
             if (iters % 2 != 0) throw Panic("iters must be even");
             py::gil_scoped_release nogil;
             std::lock_guard<std::recursive_mutex> lock(s.st->mu);
             s.st->prepare();
             check(lbm_iterate(s.st->h, iters));
             s.st->iteration += (uint64_t)iters;
           })
      .def("_read_back",
           [](Simulation& s) {
             py::gil_scoped_release nogil;
             std::lock_guard<std::recursive_mutex> lock(s.st->mu);
             s.st->read_back();
           })
      .def("_fluid_device",
           [](const Simulation& s) {
             // Device addresses of rho [N] and vel [N, D], current after each iterate call.
             void *rho = nullptr, *vel = nullptr;
             check(lbm_fluid_device(s.st->h, &rho, &vel));
             return py::make_tuple(reinterpret_cast<uintptr_t>(rho), reinterpret_cast<uintptr_t>(vel));
           })
      .def("_set_omega_field",
           [](Simulation& s, uintptr_t field) {
             // Per-cell omega+ (device address of N floats, kept alive by the caller); 0 clears it.
             std::lock_guard<std::recursive_mutex> lock(s.st->mu);
             check(lbm_set_omega_field(s.st->h, reinterpret_cast<const float*>(field)));
           })
      .def("_iterate_closure",
           [](Simulation& s, int64_t iters, int64_t every, uintptr_t params, uintptr_t params_bf16,
              uintptr_t flags, py::array_t<float, py::array::c_style | py::array::forcecast> norm,
              float tau0, float gain, float max_dtau, uintptr_t omega) {
             // Steps of a 2D run whose relaxation field the learned closure refreshes every
             // `every` steps (lbm_closure_relaxation on the simulation's stream, then `every`
             // steps), the whole loop issued from here so the GPU never waits on Python.
             // Pointers are device addresses the caller keeps alive; omega stays installed as the
             // simulation's field.
             SimState& st = *s.st;
             if (st.dim != 2 || st.q != 9) throw py::value_error("the closure drives D2Q9 runs");
             if (every <= 0 || every % 2 != 0 || iters % every != 0)
               throw py::value_error("iters must be a multiple of an even closure interval");
             if (norm.size() != 8) throw py::value_error("norm must hold 8 floats");
             std::array<float, 8> nm;
             std::copy(norm.data(), norm.data() + 8, nm.begin());
             py::gil_scoped_release nogil;
             std::lock_guard<std::recursive_mutex> lock(st.mu);
             st.prepare();
             void *rho = nullptr, *vel = nullptr, *stream = nullptr;
             check(lbm_fluid_device(st.h, &rho, &vel));
             check(lbm_stream(st.h, &stream));
             float* om = reinterpret_cast<float*>(omega);
             check(lbm_set_omega_field(st.h, om));
             for (int64_t done = 0; done < iters; done += every) {
               check(lbm_closure_relaxation(
                   reinterpret_cast<const float*>(params),
                   reinterpret_cast<const uint16_t*>(params_bf16), static_cast<const float*>(rho),
                   static_cast<const float*>(vel), reinterpret_cast<const int32_t*>(flags),
                   st.counts[0], st.counts[1], nm.data(), tau0, gain, max_dtau, om, stream));
               check(lbm_iterate(st.h, every));
               st.iteration += (uint64_t)every;
             }
           })
      .def("_launch_counts",
           [](const Simulation& s) {
             // AA step launches so far: (direct kernel, TMA-staged kernel).
             int64_t direct = 0, staged = 0;
             check(lbm_launch_counts(s.st->h, &direct, &staged));
             return py::make_tuple(direct, staged);
           })
      .def("_synchronize", [](const Simulation& s) { check(lbm_synchronize(s.st->h)); })
      .def("_stream", [](const Simulation& s) {
        void* p = nullptr;
        check(lbm_stream(s.st->h, &p));
        return reinterpret_cast<uintptr_t>(p);
      });
}
