// The reference's host-array C interface (include/wgpu_nufft.h) over the
// device plans: capi/src/lib.rs, plan.rs, cache.rs, adapter.rs of wgpuNUFFT.
//
// A host plan keeps its device plan, device copies of the points, and staging
// buffers; setpts converts and uploads the points and bins them once;
// execute uploads the input, runs the device plan on the library's stream
// and copies the output back, then returns. Type-3 plans are built at setpts
// from the bounds of the points and rebuilt only when later points leave
// them (capi/src/plan.rs:353-397). The one-call functions keep the four most
// recently used plans (capi/src/cache.rs:10). There is no CPU engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <list>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/wgpu_nufft.h"
#include "plan.h"
#include "type3.h"
#include "capi_io.h"
#include "util.h"

using b200nufft::DeviceBuffer;
using b200nufft::NufftFailure;
using b200nufft::HostScalar;
using b200nufft::capi_gather_points;
using b200nufft::capi_convert_values;
using b200nufft::capi_convert_back;
using b200nufft::capi_key_value;

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr size_t kCacheSize = 4;

enum class Data { F32, F64 };

// A return code and message for the reference's error classes.
struct CapiError {
  int code;
  std::string message;
};

int code_for(int status) {
  switch (status) {
    case B200NUFFT_INVALID_ARGUMENT:
    case B200NUFFT_INPUT_LENGTH:
    case B200NUFFT_GPU_EXECUTION_UNAVAILABLE:
    case B200NUFFT_GPU_BUFFER_ALIAS_UNSUPPORTED:
    case B200NUFFT_GPU_DEVICE_MISMATCH:
      return WGPU_NUFFT_ERROR_INVALID_ARGUMENT;
    case B200NUFFT_DEVICE_ERROR:
    case B200NUFFT_DEVICE_ALLOCATION_FAILED:
    case B200NUFFT_DEVICE_TIMEOUT:
    case B200NUFFT_FFT_EXECUTION_FAILED:
      return WGPU_NUFFT_ERROR_GPU;
    case B200NUFFT_INTERNAL:
      return WGPU_NUFFT_ERROR_INTERNAL;
    default:
      return WGPU_NUFFT_ERROR_PLAN;
  }
}

template <typename F>
int call(F&& body) {
  try {
    body();
    return WGPU_NUFFT_SUCCESS;
  } catch (const CapiError& e) {
    b200nufft::set_last_error(e.message);
    return e.code;
  } catch (const NufftFailure& f) {
    b200nufft::set_last_error(f.message);
    return code_for(f.code);
  } catch (const std::bad_alloc&) {
    b200nufft::set_last_error("host allocation failed");
    return WGPU_NUFFT_ERROR_INTERNAL;
  } catch (...) {
    b200nufft::set_last_error("internal error");
    return WGPU_NUFFT_ERROR_INTERNAL;
  }
}

[[noreturn]] void invalid(const std::string& message) {
  throw CapiError{WGPU_NUFFT_ERROR_INVALID_ARGUMENT, message};
}

std::string field_text(const char* bytes, size_t size, const char* name) {
  const void* end = std::memchr(bytes, 0, size);
  if (!end) invalid(std::string(name) + " must end with a NUL within its " + std::to_string(size) + " bytes");
  std::string text(bytes, static_cast<const char*>(end));
  const auto first = text.find_first_not_of(" \t\r\n");
  if (first == std::string::npos) return "";
  const auto last = text.find_last_not_of(" \t\r\n");
  return text.substr(first, last - first + 1);
}

std::string field_trim(const std::string& text) {
  const auto first = text.find_first_not_of(" \t\r\n");
  if (first == std::string::npos) return "";
  return text.substr(first, text.find_last_not_of(" \t\r\n") - first + 1);
}

std::string lower(std::string s) {
  for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  return s;
}

// A PCI address [domain:]bus:device[.function], each part 1 to 8 hex
// digits (PciAddress::parse, capi/src/adapter.rs:78-101).
struct PciAddress {
  uint32_t domain = 0, bus = 0, device = 0, function = 0;
  bool has_function = false;
  bool operator==(const PciAddress& o) const {
    return domain == o.domain && bus == o.bus && device == o.device &&
           has_function == o.has_function && function == o.function;
  }
  // An address without a function names every function of the device.
  bool matches(const PciAddress& o) const {
    return domain == o.domain && bus == o.bus && device == o.device &&
           (!has_function || !o.has_function || function == o.function);
  }
  std::string text() const {
    char buffer[40];
    if (has_function) {
      std::snprintf(buffer, sizeof(buffer), "%04x:%02x:%02x.%x", domain, bus, device, function);
    } else {
      std::snprintf(buffer, sizeof(buffer), "%04x:%02x:%02x", domain, bus, device);
    }
    return buffer;
  }
};

bool parse_hex(const std::string& part, uint32_t& value) {
  if (part.empty() || part.size() > 8) return false;
  value = 0;
  for (char c : part) {
    if (!std::isxdigit(static_cast<unsigned char>(c))) return false;
    value = value * 16 + static_cast<uint32_t>(std::isdigit(static_cast<unsigned char>(c))
                                                   ? c - '0'
                                                   : std::tolower(static_cast<unsigned char>(c)) - 'a' + 10);
  }
  return true;
}

bool parse_pci(std::string text, PciAddress& out) {
  const auto first = text.find_first_not_of(" \t\r\n");
  if (first == std::string::npos) return false;
  text = text.substr(first, text.find_last_not_of(" \t\r\n") - first + 1);
  PciAddress a;
  const auto dot = text.find('.');
  if (dot != std::string::npos) {
    if (!parse_hex(text.substr(dot + 1), a.function)) return false;
    a.has_function = true;
    text = text.substr(0, dot);
  }
  std::vector<std::string> parts;
  size_t from = 0;
  for (;;) {
    const auto colon = text.find(':', from);
    parts.push_back(text.substr(from, colon == std::string::npos ? std::string::npos : colon - from));
    if (colon == std::string::npos) break;
    from = colon + 1;
  }
  if (parts.size() == 3) {
    if (!parse_hex(parts[0], a.domain) || !parse_hex(parts[1], a.bus) || !parse_hex(parts[2], a.device)) return false;
  } else if (parts.size() == 2) {
    if (!parse_hex(parts[0], a.bus) || !parse_hex(parts[1], a.device)) return false;
  } else {
    return false;
  }
  out = a;
  return true;
}

// The adapter the options select; all unset picks the first CUDA device
// (AdapterSelection, capi/src/adapter.rs:127-169).
struct AdapterSelection {
  std::string name;
  bool has_pci = false;
  PciAddress pci;
  int32_t index = 0;  // position among the matches, from 1; 0 for none
  bool is_default() const { return name.empty() && !has_pci && index == 0; }
  bool operator==(const AdapterSelection& o) const {
    return name == o.name && has_pci == o.has_pci && (!has_pci || pci == o.pci) && index == o.index;
  }
  std::string text() const {
    std::vector<std::string> parts;
    if (!name.empty()) parts.push_back("name \"" + name + "\"");
    if (has_pci) parts.push_back("PCI bus ID " + pci.text());
    if (index > 0) parts.push_back("index " + std::to_string(index));
    if (parts.empty()) return "no adapter";
    std::string out = parts[0];
    for (size_t i = 1; i < parts.size(); ++i) out += ", " + parts[i];
    return out;
  }
};

struct AdapterEntry {
  std::string name;
  std::string pci;  // as the device reports it; may be empty
};

bool selection_matches(const AdapterSelection& sel, const AdapterEntry& entry) {
  if (!sel.name.empty() && lower(field_trim(entry.name)) != lower(sel.name)) return false;
  if (sel.has_pci) {
    PciAddress found;
    if (!parse_pci(entry.pci, found) || !sel.pci.matches(found)) return false;
  }
  return true;
}

std::string describe(const std::vector<AdapterEntry>& list, const std::vector<size_t>& positions) {
  if (positions.empty()) return "none";
  std::string out;
  for (size_t i = 0; i < positions.size(); ++i) {
    const AdapterEntry& e = list[positions[i]];
    if (i) out += "; ";
    out += std::to_string(positions[i] + 1) + ". " + e.name + " (CUDA, DiscreteGpu";
    if (!e.pci.empty()) out += ", " + e.pci;
    out += ")";
  }
  return out;
}

// The list position the selection names: the index counts the matches in
// list order; without an index the matches must be one adapter
// (resolve, capi/src/adapter.rs:175-207). CUDA lists each GPU once.
size_t resolve_adapter(const std::vector<AdapterEntry>& list, const AdapterSelection& sel) {
  std::vector<size_t> matches, all;
  for (size_t i = 0; i < list.size(); ++i) {
    all.push_back(i);
    if (selection_matches(sel, list[i])) matches.push_back(i);
  }
  const auto not_found = [&] {
    return CapiError{WGPU_NUFFT_ERROR_GPU_UNAVAILABLE,
                     "no GPU adapter matches " + sel.text() + "; the adapters are " + describe(list, all)};
  };
  if (sel.index > 0) {
    if (static_cast<size_t>(sel.index) > matches.size()) throw not_found();
    return matches[static_cast<size_t>(sel.index) - 1];
  }
  if (matches.empty()) throw not_found();
  if (matches.size() > 1) {
    invalid(std::to_string(matches.size()) + " CUDA adapters match " + sel.text() + ": " + describe(list, matches) +
            "; set adapter_index or adapter_pci_bus_id to choose one");
  }
  return matches.front();
}

AdapterSelection selection_of(const wgpu_nufft_opts& opts) {
  if (opts.adapter_index < 0) invalid("adapter_index must not be negative, not " + std::to_string(opts.adapter_index));
  AdapterSelection sel;
  sel.name = field_text(opts.adapter_name, sizeof(opts.adapter_name), "adapter_name");
  const std::string pci = field_text(opts.adapter_pci_bus_id, sizeof(opts.adapter_pci_bus_id), "adapter_pci_bus_id");
  if (!pci.empty()) {
    if (!parse_pci(pci, sel.pci)) {
      invalid("adapter_pci_bus_id \"" + pci + "\" is not a PCI address such as 0000:01:00.0");
    }
    sel.has_pci = true;
  }
  sel.index = opts.adapter_index;
  return sel;
}

struct Spec {
  int kind = 1;
  int dim = 1;
  std::vector<int64_t> modes;
  int isign = 1;
  int64_t ntrans = 1;
  double eps = 1e-6;
  Data data = Data::F64;
  int32_t backend = 0;
  int32_t precision = 0;
  int32_t mode_order = 0;
  double sigma = 0.0;
  AdapterSelection adapter;
  bool operator==(const Spec& o) const {
    return kind == o.kind && dim == o.dim && modes == o.modes && isign == o.isign &&
           ntrans == o.ntrans && eps == o.eps && data == o.data && backend == o.backend &&
           precision == o.precision && mode_order == o.mode_order && sigma == o.sigma &&
           adapter == o.adapter;
  }
};

Spec make_spec(int32_t kind, int32_t dim, const int64_t* n_modes, int32_t isign, int64_t ntrans,
               double eps, Data data, const wgpu_nufft_opts* opts_in) {
  wgpu_nufft_opts opts;
  if (opts_in) opts = *opts_in; else std::memset(&opts, 0, sizeof(opts));
  // Opts::validate (capi/src/plan.rs:101-125).
  if (opts.backend < WGPU_NUFFT_BACKEND_AUTO || opts.backend > WGPU_NUFFT_BACKEND_CPU) {
    invalid("unknown backend option " + std::to_string(opts.backend));
  }
  if (opts.precision < WGPU_NUFFT_PRECISION_AUTO || opts.precision > WGPU_NUFFT_PRECISION_F32) {
    invalid("unknown precision option " + std::to_string(opts.precision));
  }
  if (opts.mode_order < 0 || opts.mode_order > 1) invalid("unknown mode order option " + std::to_string(opts.mode_order));
  if (opts.threads < 0) invalid("threads must not be negative");
  if (!(opts.sigma == 0.0 || (std::isfinite(opts.sigma) && opts.sigma > 1.0))) {
    invalid("sigma must be 0 (the default) or a finite value above 1");
  }
  Spec s;
  s.adapter = selection_of(opts);
  if (kind < 1 || kind > 3) invalid("type must be 1, 2 or 3, not " + std::to_string(kind));
  if (dim < 1 || dim > 8) invalid("dim must be between 1 and 8, not " + std::to_string(dim));
  s.kind = kind;
  s.dim = dim;
  if (kind != 3) {
    if (!n_modes) invalid("n_modes is null");
    for (int a = 0; a < dim; ++a) {
      if (n_modes[a] < 1) invalid("mode counts must be positive, not " + std::to_string(n_modes[a]));
      s.modes.push_back(n_modes[a]);
    }
  }
  if (ntrans < 1) invalid("ntrans must be positive, not " + std::to_string(ntrans));
  if (!(std::isfinite(eps) && eps > 0.0)) invalid("eps must be positive and finite");
  s.isign = isign >= 0 ? 1 : -1;
  s.ntrans = ntrans;
  s.eps = eps;
  s.data = data;
  s.backend = opts.backend;
  s.precision = opts.precision;
  s.mode_order = opts.mode_order;
  s.sigma = opts.sigma;
  return s;
}

// Spec::gpu_precision (capi/src/plan.rs:246-259) on a GPU with native f64.
int gpu_precision(const Spec& s) {
  if (s.precision == WGPU_NUFFT_PRECISION_F32 ||
      (s.precision == WGPU_NUFFT_PRECISION_AUTO && s.data == Data::F32)) {
    return B200NUFFT_PRECISION_F32;
  }
  if (s.precision == WGPU_NUFFT_PRECISION_DF64) return B200NUFFT_PRECISION_DF64;
  return B200NUFFT_PRECISION_F64;
}

// ---------------------------------------------------------------------------
// The process's device (capi/src/gpu.rs:86): chosen by the first GPU plan.

std::mutex g_device_mutex;
int g_device = -1;
AdapterSelection g_device_selection;

// The CUDA devices in ordinal order; position i is device i.
std::vector<AdapterEntry> cuda_devices() {
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess) {
    cudaGetLastError();
    return {};
  }
  std::vector<AdapterEntry> devices;
  for (int d = 0; d < count; ++d) {
    cudaDeviceProp prop;
    AdapterEntry entry;
    if (cudaGetDeviceProperties(&prop, d) == cudaSuccess) {
      entry.name = prop.name;
    } else {
      cudaGetLastError();
      entry.name = "CUDA device " + std::to_string(d);
    }
    char bus[32] = {0};
    PciAddress address;
    if (cudaDeviceGetPCIBusId(bus, sizeof(bus), d) == cudaSuccess && parse_pci(bus, address)) {
      entry.pci = address.text();
    } else {
      cudaGetLastError();
    }
    devices.push_back(entry);
  }
  return devices;
}

int select_device(const AdapterSelection& sel) {
  std::lock_guard<std::mutex> lock(g_device_mutex);
  if (g_device >= 0 && (sel.is_default() || sel == g_device_selection)) return g_device;
  const auto devices = cuda_devices();
  if (devices.empty()) throw CapiError{WGPU_NUFFT_ERROR_GPU_UNAVAILABLE, "no GPU adapter: no CUDA device is available"};
  const int chosen = sel.is_default() ? 0 : static_cast<int>(resolve_adapter(devices, sel));
  if (g_device >= 0 && chosen != g_device) {
    invalid("the shared GPU device was created on another adapter; call wgpu_nufft_shutdown() first");
  }
  g_device = chosen;
  g_device_selection = sel;
  return chosen;
}

// ---------------------------------------------------------------------------

// A non-blocking stream for the input upload of execute, so that the copy
// overlaps the bin sort that set_points left running on the default stream;
// the plan's kernels wait for it through `uploaded`.
struct UploadStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t uploaded = nullptr;
  int device = -1;
  void ensure(int dev) {
    if (stream) return;
    b200nufft::check_cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "create upload stream");
    b200nufft::check_cuda(cudaEventCreateWithFlags(&uploaded, cudaEventDisableTiming), "create upload event");
    device = dev;
  }
  UploadStream() = default;
  UploadStream(const UploadStream&) = delete;
  UploadStream& operator=(const UploadStream&) = delete;
  ~UploadStream() {
    if (!stream) return;
    int current = 0;
    cudaGetDevice(&current);
    cudaSetDevice(device);
    cudaEventDestroy(uploaded);
    cudaStreamDestroy(stream);
    cudaSetDevice(current);
  }
};

struct HostPlan {
  Spec spec;
  int precision = B200NUFFT_PRECISION_F64;
  int device = 0;
  int64_t mode_count = 1;
  std::unique_ptr<b200nufft::NufftPlan> plan12;
  std::unique_ptr<b200nufft::Type3Plan> plan3;
  std::vector<double> source_lo, source_hi, target_lo, target_hi;
  DeviceBuffer points, targets, input, output, staging, checks;
  UploadStream upload;
  int64_t point_count = -1;
  int64_t target_count = 0;
};

size_t scalar_bytes(int precision) { return precision == B200NUFFT_PRECISION_F32 ? 4 : 8; }

b200nufft_type3_config type3_config(const HostPlan& p, const std::vector<double>& slo,
                                    const std::vector<double>& shi, const std::vector<double>& tlo,
                                    const std::vector<double>& thi) {
  b200nufft_type3_config c;
  std::memset(&c, 0, sizeof(c));
  c.dimensions = p.spec.dim;
  c.batch = p.spec.ntrans;
  c.eps = p.spec.eps;
  c.isign = p.spec.isign;
  c.sigma = p.spec.sigma;
  c.precision = p.precision;
  c.device = p.device;
  for (int a = 0; a < p.spec.dim; ++a) {
    c.source_lower[a] = slo[a];
    c.source_upper[a] = shi[a];
    c.target_lower[a] = tlo[a];
    c.target_upper[a] = thi[a];
  }
  return c;
}

std::unique_ptr<HostPlan> make_host_plan(const Spec& spec) {
  if (spec.backend == WGPU_NUFFT_BACKEND_CPU) {
    throw CapiError{WGPU_NUFFT_ERROR_PLAN,
                    "this library has no CPU engine; use the GPU or automatic backend"};
  }
  auto plan = std::make_unique<HostPlan>();
  plan->spec = spec;
  plan->precision = gpu_precision(spec);
  plan->device = select_device(spec.adapter);
  b200nufft::check_cuda(cudaSetDevice(plan->device), "select device");
  if (spec.kind != 3) {
    if (spec.dim > B200NUFFT_MAX_DIMENSIONS) {
      throw NufftFailure{B200NUFFT_GPU_DIMENSIONS_UNSUPPORTED, "GPU plans support 1 to 8 dimensions"};
    }
    b200nufft_config c;
    b200nufft_default_config(&c);
    c.type = spec.kind;
    c.dimensions = spec.dim;
    for (int a = 0; a < spec.dim; ++a) {
      c.n_modes[a] = spec.modes[a];
      plan->mode_count *= spec.modes[a];
    }
    c.batch = spec.ntrans;
    c.eps = spec.eps;
    c.isign = spec.isign;
    c.mode_order = spec.mode_order;
    c.sigma = spec.sigma;
    c.precision = plan->precision;
    c.device = plan->device;
    plan->plan12 = std::make_unique<b200nufft::NufftPlan>(c, true);
  } else {
    if (spec.dim > B200NUFFT_MAX_TYPE3_DIMENSIONS) {
      throw NufftFailure{B200NUFFT_GPU_DIMENSIONS_UNSUPPORTED, "GPU type-3 plans support 1 to 3 dimensions"};
    }
    // The parts of the configuration that do not depend on the points are
    // checked now, on unit intervals; the kept plan is built at setpts.
    const std::vector<double> unit_lo(spec.dim, -1.0), unit_hi(spec.dim, 1.0);
    b200nufft::Type3Plan check(type3_config(*plan, unit_lo, unit_hi, unit_lo, unit_hi));
  }
  return plan;
}

bool storage_matches(int precision, HostScalar scalar) {
  return (precision == B200NUFFT_PRECISION_F32 && scalar == HostScalar::F32) ||
         (precision == B200NUFFT_PRECISION_F64 && scalar == HostScalar::F64);
}

template <typename T>
constexpr HostScalar host_scalar() {
  return std::is_same<T, float>::value ? HostScalar::F32 : HostScalar::F64;
}

// A point set as the caller passes it: one array per axis or one point-major array.
template <typename T>
struct HostPoints {
  int64_t count = 0;
  const T* axes[3] = {nullptr, nullptr, nullptr};
  const T* interleaved = nullptr;
  const char* const* names = nullptr;  // per-axis argument names, or the point-major one
};

template <typename T>
void validate_points(const HostPoints<T>& h, int dim) {
  if (h.count < 0) invalid("M must not be negative");
  if (h.count == 0) return;
  if (h.names && dim <= 3 && !h.interleaved) {
    for (int a = 0; a < dim; ++a) {
      if (!h.axes[a]) invalid(std::string(h.names[a]) + " is null");
    }
  } else if (!h.interleaved) {
    invalid("the point array is null");
  }
}

template <typename T>
double host_coordinate(const HostPoints<T>& h, int dim, int64_t i, int a) {
  return h.interleaved ? static_cast<double>(h.interleaved[i * dim + a]) : static_cast<double>(h.axes[a][i]);
}

// Copies the caller's coordinates to `staging` as they are and converts them
// to point-major storage in `out` on the device.
template <typename T>
void upload_points(HostPlan& p, const HostPoints<T>& h, DeviceBuffer& out, int check,
                   unsigned long long* first_bad, unsigned long long* bounds, size_t staging_offset) {
  const int dim = p.spec.dim;
  const size_t bytes = static_cast<size_t>(h.count) * dim * sizeof(T);
  const size_t storage = static_cast<size_t>(h.count) * dim * scalar_bytes(p.precision);
  void* dst = out.reserve(std::max<size_t>(storage, 16), "coordinates");
  if (h.count == 0) return;
  unsigned char* stage = static_cast<unsigned char*>(p.staging.get()) + staging_offset;
  if (h.interleaved) {
    b200nufft::check_cuda(cudaMemcpyAsync(stage, h.interleaved, bytes, cudaMemcpyHostToDevice, nullptr),
                          "copy points");
    capi_gather_points(host_scalar<T>(), stage, 1, dim, dim, h.count, p.precision, check, dst, first_bad, bounds,
                       nullptr);
  } else {
    for (int a = 0; a < dim; ++a) {
      b200nufft::check_cuda(cudaMemcpyAsync(stage + a * h.count * sizeof(T), h.axes[a], h.count * sizeof(T),
                                            cudaMemcpyHostToDevice, nullptr),
                            "copy points");
    }
    capi_gather_points(host_scalar<T>(), stage, h.count, 1, dim, h.count, p.precision, check, dst, first_bad,
                       bounds, nullptr);
  }
}

double rounded(double v, int precision) {
  return precision == B200NUFFT_PRECISION_F32 ? static_cast<double>(static_cast<float>(v)) : v;
}

std::string number(double v) {
  char buffer[64];
  std::snprintf(buffer, sizeof(buffer), "%.17g", v);
  return buffer;
}

// Plan::set_points (capi/src/plan.rs:478-523) with the checks of
// check_type12_points / check_finite (:524-545) on the device.
template <typename T>
void set_points(HostPlan& p, const HostPoints<T>& pts, const HostPoints<T>& tgs) {
  b200nufft::check_cuda(cudaSetDevice(p.device), "select device");
  const int dim = p.spec.dim;
  validate_points(pts, dim);
  const bool type3 = p.spec.kind == 3;
  if (type3) validate_points(tgs, dim);
  p.point_count = -1;
  const size_t point_bytes = static_cast<size_t>(pts.count) * dim * sizeof(T);
  const size_t target_bytes = type3 ? static_cast<size_t>(tgs.count) * dim * sizeof(T) : 0;
  const size_t target_offset = (point_bytes + 255) / 256 * 256;
  p.staging.reserve(std::max<size_t>(target_offset + target_bytes, 16), "host copies");
  // checks: [0] first bad point element, [1] first bad target element,
  // [2 .. 2 + 2 dim) point bounds, [2 + 2 dim .. 2 + 4 dim) target bounds.
  unsigned long long init[2 + 4 * 8];
  init[0] = init[1] = ~0ull;
  for (int a = 0; a < dim; ++a) {
    init[2 + 2 * a] = init[2 + 2 * dim + 2 * a] = ~0ull;
    init[3 + 2 * a] = init[3 + 2 * dim + 2 * a] = 0ull;
  }
  unsigned long long* checks = static_cast<unsigned long long*>(p.checks.reserve(sizeof(init), "checks"));
  b200nufft::check_cuda(cudaMemcpyAsync(checks, init, sizeof(init), cudaMemcpyHostToDevice, nullptr), "reset checks");
  upload_points(p, pts, p.points, type3 ? 1 : 0, checks, type3 ? checks + 2 : nullptr, 0);
  if (type3) upload_points(p, tgs, p.targets, 1, checks + 1, checks + 2 + 2 * dim, target_offset);
  unsigned long long result[2 + 4 * 8];
  b200nufft::check_cuda(cudaMemcpy(result, checks, sizeof(result), cudaMemcpyDeviceToHost), "read checks");
  if (type3 && result[1] != ~0ull) {
    const int64_t i = static_cast<int64_t>(result[1] / dim);
    invalid("target " + std::to_string(i) + " has a coordinate that is not finite on axis " +
            std::to_string(result[1] % dim));
  }
  if (result[0] != ~0ull) {
    const int64_t i = static_cast<int64_t>(result[0] / dim);
    const int a = static_cast<int>(result[0] % dim);
    if (type3) {
      invalid("point " + std::to_string(i) + " has a coordinate that is not finite on axis " + std::to_string(a));
    }
    invalid("point " + std::to_string(i) + " has coordinate " +
            number(rounded(host_coordinate(pts, dim, i, a), p.precision)) + " on axis " + std::to_string(a) +
            ", outside [-3*pi, 3*pi]");
  }
  if (!type3) {
    p.plan12->set_points(pts.count, p.points.get(), nullptr);
  } else {
    // The smallest interval per axis holding every point, [0, 0] without any
    // (intervals, capi/src/plan.rs:377-397).
    std::vector<double> slo(dim), shi(dim), tlo(dim), thi(dim);
    for (int a = 0; a < dim; ++a) {
      const bool any_s = pts.count > 0, any_t = tgs.count > 0;
      slo[a] = any_s ? capi_key_value(result[2 + 2 * a]) : 0.0;
      shi[a] = any_s ? capi_key_value(result[3 + 2 * a]) : 0.0;
      tlo[a] = any_t ? capi_key_value(result[2 + 2 * dim + 2 * a]) : 0.0;
      thi[a] = any_t ? capi_key_value(result[3 + 2 * dim + 2 * a]) : 0.0;
    }
    bool contained = p.plan3 != nullptr;
    for (int a = 0; contained && a < dim; ++a) {
      contained = p.source_lo[a] <= slo[a] && shi[a] <= p.source_hi[a] && p.target_lo[a] <= tlo[a] &&
                  thi[a] <= p.target_hi[a];
    }
    if (!contained) {
      p.plan3.reset();
      p.plan3 = std::make_unique<b200nufft::Type3Plan>(type3_config(p, slo, shi, tlo, thi));
      p.source_lo = slo;
      p.source_hi = shi;
      p.target_lo = tlo;
      p.target_hi = thi;
    }
    p.plan3->set_points(pts.count, p.points.get(), tgs.count, p.targets.get(), nullptr);
  }
  p.point_count = pts.count;
  p.target_count = type3 ? tgs.count : 0;
}

void lengths(const HostPlan& p, int64_t& in_complex, int64_t& out_complex) {
  if (p.point_count < 0) invalid("set the points before executing the plan");
  const int64_t nt = p.spec.ntrans;
  switch (p.spec.kind) {
    case 1: in_complex = p.point_count * nt; out_complex = p.mode_count * nt; break;
    case 2: in_complex = p.mode_count * nt; out_complex = p.point_count * nt; break;
    default: in_complex = p.point_count * nt; out_complex = p.target_count * nt; break;
  }
}

// Plan::execute (capi/src/plan.rs:547-570): the input copied as it is and
// checked on the device; the output copied back when every value was finite.
template <typename T>
void execute(HostPlan& p, const T* in, T* out, const char* in_name, const char* out_name) {
  b200nufft::check_cuda(cudaSetDevice(p.device), "select device");
  int64_t in_complex, out_complex;
  lengths(p, in_complex, out_complex);
  const int64_t in_scalars = 2 * in_complex, out_scalars = 2 * out_complex;
  if (in_scalars > 0 && !in) invalid(std::string(in_name) + " is null");
  if (out_scalars > 0 && !out) invalid(std::string(out_name) + " is null");
  const HostScalar scalar = host_scalar<T>();
  const bool direct = storage_matches(p.precision, scalar);
  const size_t in_storage = static_cast<size_t>(in_scalars) * scalar_bytes(p.precision);
  const size_t out_storage = static_cast<size_t>(out_scalars) * scalar_bytes(p.precision);
  void* d_in = p.input.reserve(std::max<size_t>(in_storage, 16), "input");
  void* d_out = p.output.reserve(std::max<size_t>(out_storage, 16), "output");
  if (!direct) {
    p.staging.reserve(std::max<size_t>(static_cast<size_t>(std::max(in_scalars, out_scalars)) * sizeof(T), 16),
                      "host copies");
  }
  unsigned long long* checks = static_cast<unsigned long long*>(p.checks.reserve(16 * sizeof(unsigned long long), "checks"));
  // The upload and its checks run beside the sort of set_points (the previous
  // execute ended with a synchronous read, and set_points' own copies were
  // read back, so nothing in flight uses these buffers).
  p.upload.ensure(p.device);
  cudaStream_t upload = p.upload.stream;
  b200nufft::check_cuda(cudaMemsetAsync(checks, 0xFF, sizeof(unsigned long long), upload), "reset checks");
  if (in_scalars > 0) {
    void* landing = direct ? d_in : p.staging.get();
    b200nufft::check_cuda(cudaMemcpyAsync(landing, in, static_cast<size_t>(in_scalars) * sizeof(T),
                                          cudaMemcpyHostToDevice, upload),
                          "copy input");
    capi_convert_values(scalar, landing, in_scalars, p.precision, direct ? nullptr : d_in, checks, upload);
  }
  b200nufft::check_cuda(cudaEventRecord(p.upload.uploaded, upload), "record upload");
  b200nufft::check_cuda(cudaStreamWaitEvent(nullptr, p.upload.uploaded, 0), "wait for upload");
  if (p.spec.kind != 3) {
    p.plan12->execute(p.spec.ntrans, d_in, d_out, nullptr);
  } else {
    p.plan3->execute(p.spec.ntrans, d_in, d_out, nullptr);
  }
  unsigned long long first_bad = 0;
  b200nufft::check_cuda(cudaMemcpy(&first_bad, checks, sizeof(first_bad), cudaMemcpyDeviceToHost), "read checks");
  if (p.spec.kind != 3) p.plan12->synchronize(nullptr);
  if (first_bad != ~0ull) {
    invalid("the input holds a value that is not finite at complex index " + std::to_string(first_bad / 2));
  }
  if (out_scalars > 0) {
    const void* source = d_out;
    if (!direct) {
      capi_convert_back(p.precision, d_out, out_scalars, scalar, p.staging.get(), nullptr);
      source = p.staging.get();
    }
    b200nufft::check_cuda(cudaMemcpy(out, source, static_cast<size_t>(out_scalars) * sizeof(T),
                                     cudaMemcpyDeviceToHost),
                          "read output");
  }
}

// ---------------------------------------------------------------------------
// The kept plans of the one-call functions.

std::mutex g_cache_mutex;
std::list<std::unique_ptr<HostPlan>> g_cache;

template <typename T>
int one_call(int kind, int dim, int64_t m, const T* const* axes, int32_t isign, double eps,
             const int64_t* modes, int64_t n, const T* const* target_axes, const T* input, T* output,
             const wgpu_nufft_opts* opts, Data data) {
  return call([&] {
    const Spec spec = make_spec(kind, dim, modes, isign, 1, eps, data, opts);
    static const char* const xyz[] = {"x", "y", "z"};
    static const char* const stu[] = {"s", "t", "u"};
    HostPoints<T> pts, tgs;
    pts.count = m;
    pts.names = xyz;
    for (int a = 0; a < dim; ++a) pts.axes[a] = axes[a];
    if (kind == 3) {
      if (n < 0) invalid("N must not be negative");
      tgs.count = n;
      tgs.names = stu;
      for (int a = 0; a < dim; ++a) tgs.axes[a] = target_axes[a];
    }
    // The arrays are checked before a plan is made or taken from the cache.
    validate_points(pts, dim);
    if (kind == 3) validate_points(tgs, dim);
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    auto found = std::find_if(g_cache.begin(), g_cache.end(),
                              [&](const std::unique_ptr<HostPlan>& p) { return p->spec == spec; });
    std::unique_ptr<HostPlan> plan;
    if (found != g_cache.end()) {
      plan = std::move(*found);
      g_cache.erase(found);
    } else {
      plan = make_host_plan(spec);
    }
    // The plan stays kept whether or not the call succeeds.
    struct Keep {
      std::unique_ptr<HostPlan>& plan;
      ~Keep() {
        g_cache.push_front(std::move(plan));
        while (g_cache.size() > kCacheSize) g_cache.pop_back();
      }
    } keep{plan};
    set_points(*plan, pts, tgs);
    execute(*plan, input, output, kind == 2 ? "f" : "c", kind == 2 ? "c" : "f");
  });
}

}  // namespace

namespace {

// What both opaque handle types point to, so that a plan passed to the
// other family's functions is recognised and refused (capi/src/lib.rs).
struct PlanHandle {
  Data data = Data::F64;
  std::unique_ptr<HostPlan> plan;
};


template <typename T>
constexpr Data data_of() {
  return std::is_same<T, float>::value ? Data::F32 : Data::F64;
}

template <typename T>
HostPlan& host(void* handle) {
  auto* h = static_cast<PlanHandle*>(handle);
  if (!h || !h->plan) invalid("the plan is null");
  if (h->data != data_of<T>()) {
    invalid(std::string("the plan was made for ") + (h->data == Data::F32 ? "float" : "double") +
            " arrays; call the functions of that array type");
  }
  return *h->plan;
}

template <typename Handle>
int makeplan_impl(int32_t type, int32_t dim, const int64_t* n_modes, int32_t isign, int64_t ntrans,
                  double eps, Handle** out, const wgpu_nufft_opts* opts, Data data) {
  return call([&] {
    if (!out) invalid("the plan pointer is null");
    *out = nullptr;
    const Spec spec = make_spec(type, dim, n_modes, isign, ntrans, eps, data, opts);
    auto handle = std::make_unique<PlanHandle>();
    handle->data = data;
    handle->plan = make_host_plan(spec);
    *out = reinterpret_cast<Handle*>(handle.release());
  });
}

template <typename T>
int setpts_impl(void* handle, int64_t m, const T* x, const T* y, const T* z, int64_t n, const T* s,
                const T* t, const T* u) {
  return call([&] {
    HostPlan& p = host<T>(handle);
    if (p.spec.dim > 3) invalid("plans of more than three dimensions take their points through setpts_nd");
    static const char* const xyz[] = {"x", "y", "z"};
    static const char* const stu[] = {"s", "t", "u"};
    HostPoints<T> pts, tgs;
    pts.count = m;
    pts.names = xyz;
    pts.axes[0] = x;
    pts.axes[1] = y;
    pts.axes[2] = z;
    if (p.spec.kind == 3) {
      if (n < 0) invalid("N must not be negative");
      tgs.count = n;
      tgs.names = stu;
      tgs.axes[0] = s;
      tgs.axes[1] = t;
      tgs.axes[2] = u;
    }
    set_points(p, pts, tgs);
  });
}

template <typename T>
int setpts_nd_impl(void* handle, int64_t m, const T* points, int64_t n, const T* targets) {
  return call([&] {
    HostPlan& p = host<T>(handle);
    HostPoints<T> pts, tgs;
    pts.count = m;
    pts.interleaved = points;
    if (m > 0 && !points) invalid("points is null");
    if (p.spec.kind == 3) {
      if (n < 0) invalid("N must not be negative");
      if (n > 0 && !targets) invalid("targets is null");
      tgs.count = n;
      tgs.interleaved = targets;
    }
    set_points(p, pts, tgs);
  });
}

template <typename T>
int execute_impl(void* handle, T* c, T* f) {
  return call([&] {
    HostPlan& p = host<T>(handle);
    if (p.spec.kind == 2) {
      execute<T>(p, f, c, "f", "c");
    } else {
      execute<T>(p, c, f, "c", "f");
    }
  });
}

int backend_of(void* handle) {
  auto* h = static_cast<PlanHandle*>(handle);
  return h && h->plan ? WGPU_NUFFT_BACKEND_GPU : -1;
}

int precision_of(void* handle) {
  auto* h = static_cast<PlanHandle*>(handle);
  if (!h || !h->plan) return -1;
  switch (h->plan->precision) {
    case B200NUFFT_PRECISION_F32: return WGPU_NUFFT_PRECISION_F32;
    case B200NUFFT_PRECISION_DF64: return WGPU_NUFFT_PRECISION_DF64;
    default: return WGPU_NUFFT_PRECISION_F64;
  }
}

void copy_text(char* out, size_t size, const std::string& text) {
  const size_t n = std::min(size - 1, text.size());
  std::memcpy(out, text.data(), n);
  std::memset(out + n, 0, size - n);
}

}  // namespace

extern "C" {

void wgpu_nufft_default_opts(wgpu_nufft_opts* opts) {
  if (opts) std::memset(opts, 0, sizeof(*opts));
}

int wgpu_nufft_list_adapters(wgpu_nufft_adapter* adapters, int32_t capacity, int32_t* count) {
  return call([&] {
    if (!count) invalid("the count pointer is null");
    *count = 0;
    if (capacity < 0) invalid("capacity must not be negative, not " + std::to_string(capacity));
    if (capacity > 0 && !adapters) invalid("adapters is null");
    const auto devices = cuda_devices();
    for (size_t i = 0; i < devices.size() && static_cast<int32_t>(i) < capacity; ++i) {
      wgpu_nufft_adapter& a = adapters[i];
      copy_text(a.name, sizeof(a.name), devices[i].name);
      copy_text(a.backend, sizeof(a.backend), "CUDA");
      copy_text(a.device_type, sizeof(a.device_type), "DiscreteGpu");
      copy_text(a.pci_bus_id, sizeof(a.pci_bus_id), devices[i].pci);
      a.is_default = i == 0 ? 1 : 0;
    }
    *count = static_cast<int32_t>(devices.size());
  });
}

int b200nufft_resolve_adapter(const char* const* names, const char* const* pci_bus_ids, int32_t count,
                              const wgpu_nufft_opts* opts, int32_t* position) {
  return call([&] {
    if (!position) invalid("the position pointer is null");
    *position = -1;
    if (count < 0) invalid("count must not be negative, not " + std::to_string(count));
    if (count > 0 && !names) invalid("names is null");
    wgpu_nufft_opts o;
    if (opts) o = *opts; else std::memset(&o, 0, sizeof(o));
    const AdapterSelection sel = selection_of(o);
    std::vector<AdapterEntry> list;
    for (int32_t i = 0; i < count; ++i) {
      AdapterEntry e;
      e.name = names[i] ? names[i] : "";
      e.pci = pci_bus_ids && pci_bus_ids[i] ? pci_bus_ids[i] : "";
      list.push_back(e);
    }
    if (sel.is_default()) {
      if (list.empty()) throw CapiError{WGPU_NUFFT_ERROR_GPU_UNAVAILABLE, "no GPU adapter: the list is empty"};
      *position = 0;
      return;
    }
    *position = static_cast<int32_t>(resolve_adapter(list, sel));
  });
}

const char* wgpu_nufft_last_error(void) { return b200nufft::last_error(); }

const char* wgpu_nufft_version(void) { return "0.3.2"; }

const char* wgpu_nufft_gpu_name(void) {
  static std::mutex mutex;
  static std::string name;
  std::lock_guard<std::mutex> lock(mutex);
  name.clear();
  try {
    const int device = select_device(AdapterSelection{});
    const auto devices = cuda_devices();
    if (device < static_cast<int>(devices.size())) name = devices[device].name + " (CUDA)";
  } catch (...) {
    name.clear();
  }
  return name.c_str();
}

void wgpu_nufft_shutdown(void) {
  {
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    g_cache.clear();
  }
  std::lock_guard<std::mutex> lock(g_device_mutex);
  g_device = -1;
  g_device_selection = AdapterSelection{};
}

int wgpu_nufft_makeplan(int32_t type, int32_t dim, const int64_t* n_modes, int32_t isign,
                        int64_t ntrans, double eps, wgpu_nufft_plan* plan,
                        const wgpu_nufft_opts* opts) {
  return makeplan_impl(type, dim, n_modes, isign, ntrans, eps, plan, opts, Data::F64);
}
int wgpu_nufft_setpts(wgpu_nufft_plan plan, int64_t M, const double* x, const double* y,
                      const double* z, int64_t N, const double* s, const double* t, const double* u) {
  return setpts_impl<double>(plan, M, x, y, z, N, s, t, u);
}
int wgpu_nufft_setpts_nd(wgpu_nufft_plan plan, int64_t M, const double* points, int64_t N,
                         const double* targets) {
  return setpts_nd_impl<double>(plan, M, points, N, targets);
}
int wgpu_nufft_execute(wgpu_nufft_plan plan, double* c, double* f) { return execute_impl<double>(plan, c, f); }
void wgpu_nufft_destroy(wgpu_nufft_plan plan) {
  try {
    delete static_cast<PlanHandle*>(static_cast<void*>(plan));
  } catch (...) {
  }
}
int wgpu_nufft_plan_backend(wgpu_nufft_plan plan) { return backend_of(plan); }
int wgpu_nufft_plan_precision(wgpu_nufft_plan plan) { return precision_of(plan); }

int wgpu_nufftf_makeplan(int32_t type, int32_t dim, const int64_t* n_modes, int32_t isign,
                         int64_t ntrans, double eps, wgpu_nufftf_plan* plan,
                         const wgpu_nufft_opts* opts) {
  return makeplan_impl(type, dim, n_modes, isign, ntrans, eps, plan, opts, Data::F32);
}
int wgpu_nufftf_setpts(wgpu_nufftf_plan plan, int64_t M, const float* x, const float* y,
                       const float* z, int64_t N, const float* s, const float* t, const float* u) {
  return setpts_impl<float>(plan, M, x, y, z, N, s, t, u);
}
int wgpu_nufftf_setpts_nd(wgpu_nufftf_plan plan, int64_t M, const float* points, int64_t N,
                          const float* targets) {
  return setpts_nd_impl<float>(plan, M, points, N, targets);
}
int wgpu_nufftf_execute(wgpu_nufftf_plan plan, float* c, float* f) { return execute_impl<float>(plan, c, f); }
void wgpu_nufftf_destroy(wgpu_nufftf_plan plan) {
  try {
    delete static_cast<PlanHandle*>(static_cast<void*>(plan));
  } catch (...) {
  }
}
int wgpu_nufftf_plan_backend(wgpu_nufftf_plan plan) { return backend_of(plan); }
int wgpu_nufftf_plan_precision(wgpu_nufftf_plan plan) { return precision_of(plan); }

#define B200_ONE_CALL_1D(NAME, T, DATA)                                                          \
  int NAME##1d1(int64_t M, const T* x, const T* c, int32_t isign, double eps, int64_t ms, T* f,  \
                const wgpu_nufft_opts* opts) {                                                   \
    const T* ax[1] = {x};                                                                        \
    const int64_t modes[1] = {ms};                                                               \
    return one_call<T>(1, 1, M, ax, isign, eps, modes, 0, nullptr, c, f, opts, DATA);            \
  }                                                                                              \
  int NAME##1d2(int64_t M, const T* x, T* c, int32_t isign, double eps, int64_t ms, const T* f,  \
                const wgpu_nufft_opts* opts) {                                                   \
    const T* ax[1] = {x};                                                                        \
    const int64_t modes[1] = {ms};                                                               \
    return one_call<T>(2, 1, M, ax, isign, eps, modes, 0, nullptr, f, c, opts, DATA);            \
  }                                                                                              \
  int NAME##1d3(int64_t M, const T* x, const T* c, int32_t isign, double eps, int64_t N,         \
                const T* s, T* f, const wgpu_nufft_opts* opts) {                                 \
    const T* ax[1] = {x};                                                                        \
    const T* tg[1] = {s};                                                                        \
    return one_call<T>(3, 1, M, ax, isign, eps, nullptr, N, tg, c, f, opts, DATA);               \
  }

#define B200_ONE_CALL_2D(NAME, T, DATA)                                                          \
  int NAME##2d1(int64_t M, const T* x, const T* y, const T* c, int32_t isign, double eps,        \
                int64_t ms, int64_t mt, T* f, const wgpu_nufft_opts* opts) {                     \
    const T* ax[2] = {x, y};                                                                     \
    const int64_t modes[2] = {ms, mt};                                                           \
    return one_call<T>(1, 2, M, ax, isign, eps, modes, 0, nullptr, c, f, opts, DATA);            \
  }                                                                                              \
  int NAME##2d2(int64_t M, const T* x, const T* y, T* c, int32_t isign, double eps, int64_t ms,  \
                int64_t mt, const T* f, const wgpu_nufft_opts* opts) {                           \
    const T* ax[2] = {x, y};                                                                     \
    const int64_t modes[2] = {ms, mt};                                                           \
    return one_call<T>(2, 2, M, ax, isign, eps, modes, 0, nullptr, f, c, opts, DATA);            \
  }                                                                                              \
  int NAME##2d3(int64_t M, const T* x, const T* y, const T* c, int32_t isign, double eps,        \
                int64_t N, const T* s, const T* t, T* f, const wgpu_nufft_opts* opts) {          \
    const T* ax[2] = {x, y};                                                                     \
    const T* tg[2] = {s, t};                                                                     \
    return one_call<T>(3, 2, M, ax, isign, eps, nullptr, N, tg, c, f, opts, DATA);               \
  }

#define B200_ONE_CALL_3D(NAME, T, DATA)                                                          \
  int NAME##3d1(int64_t M, const T* x, const T* y, const T* z, const T* c, int32_t isign,        \
                double eps, int64_t ms, int64_t mt, int64_t mu, T* f, const wgpu_nufft_opts* opts) { \
    const T* ax[3] = {x, y, z};                                                                  \
    const int64_t modes[3] = {ms, mt, mu};                                                       \
    return one_call<T>(1, 3, M, ax, isign, eps, modes, 0, nullptr, c, f, opts, DATA);            \
  }                                                                                              \
  int NAME##3d2(int64_t M, const T* x, const T* y, const T* z, T* c, int32_t isign, double eps,  \
                int64_t ms, int64_t mt, int64_t mu, const T* f, const wgpu_nufft_opts* opts) {   \
    const T* ax[3] = {x, y, z};                                                                  \
    const int64_t modes[3] = {ms, mt, mu};                                                       \
    return one_call<T>(2, 3, M, ax, isign, eps, modes, 0, nullptr, f, c, opts, DATA);            \
  }                                                                                              \
  int NAME##3d3(int64_t M, const T* x, const T* y, const T* z, const T* c, int32_t isign,        \
                double eps, int64_t N, const T* s, const T* t, const T* u, T* f,                 \
                const wgpu_nufft_opts* opts) {                                                   \
    const T* ax[3] = {x, y, z};                                                                  \
    const T* tg[3] = {s, t, u};                                                                  \
    return one_call<T>(3, 3, M, ax, isign, eps, nullptr, N, tg, c, f, opts, DATA);               \
  }

B200_ONE_CALL_1D(wgpu_nufft, double, Data::F64)
B200_ONE_CALL_2D(wgpu_nufft, double, Data::F64)
B200_ONE_CALL_3D(wgpu_nufft, double, Data::F64)
B200_ONE_CALL_1D(wgpu_nufftf, float, Data::F32)
B200_ONE_CALL_2D(wgpu_nufftf, float, Data::F32)
B200_ONE_CALL_3D(wgpu_nufftf, float, Data::F32)

}  // extern "C"
