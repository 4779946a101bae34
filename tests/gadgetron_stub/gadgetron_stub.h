// Test-only stand-ins for the Gadgetron / gt-tomography interfaces used by
// include/cbct_gadgetron.hpp (signatures follow their use in xray/*.cpp and
// solvers/*.h).  Device arrays own cudaMalloc'd memory or view it.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <vector>

namespace boost {
using std::make_shared;
using std::shared_ptr;
}  // namespace boost

namespace Gadgetron {

template <class T, unsigned D>
struct vector_td {
  T v[D];
  vector_td() : v{} {}
  template <class... A>
  vector_td(A... a) : v{T(a)...} {}
  T& operator[](unsigned i) { return v[i]; }
  const T& operator[](unsigned i) const { return v[i]; }
};
using floatd2 = vector_td<float, 2>;
using floatd3 = vector_td<float, 3>;

// Host array: owns its elements, or views memory it does not own (the
// reference's hoCuNDArray(dims*, ptr) constructor, used for per-bin views).
template <class T>
class hoCuNDArray {
 public:
  hoCuNDArray() = default;
  explicit hoCuNDArray(const std::vector<size_t>& d) : dims_(d), own_(count(d)), ptr_(own_.data()) {}
  explicit hoCuNDArray(const std::vector<size_t>* d) : hoCuNDArray(*d) {}
  explicit hoCuNDArray(const boost::shared_ptr<std::vector<size_t>>& d) : hoCuNDArray(*d) {}
  hoCuNDArray(const std::vector<size_t>* d, T* ptr) : dims_(*d), ptr_(ptr) {}
  hoCuNDArray(const hoCuNDArray& o) : dims_(o.dims_), own_(o.ptr_, o.ptr_ + count(o.dims_)), ptr_(own_.data()) {}
  hoCuNDArray& operator=(const hoCuNDArray& o) {
    dims_ = o.dims_;
    own_.assign(o.ptr_, o.ptr_ + count(o.dims_));
    ptr_ = own_.data();
    return *this;
  }
  T* get_data_ptr() { return ptr_; }
  const T* get_data_ptr() const { return ptr_; }
  size_t get_size(size_t i) const { return i < dims_.size() ? dims_[i] : 1; }
  size_t get_number_of_dimensions() const { return dims_.size(); }
  size_t get_number_of_elements() const { return count(dims_); }
  boost::shared_ptr<std::vector<size_t>> get_dimensions() const { return boost::make_shared<std::vector<size_t>>(dims_); }
  static size_t count(const std::vector<size_t>& d) {
    return std::accumulate(d.begin(), d.end(), size_t(1), std::multiplies<size_t>());
  }
  hoCuNDArray& operator*=(T s) {
    for (size_t i = 0; i < get_number_of_elements(); ++i) ptr_[i] *= s;
    return *this;
  }

 private:
  std::vector<size_t> dims_;
  std::vector<T> own_;
  T* ptr_ = nullptr;
};

// Gadgetron's dot of two host arrays (hoCuNDArray_blas), here in double on the host.
template <class T>
T dot(hoCuNDArray<T>* a, hoCuNDArray<T>* b) {
  double s = 0.0;
  for (size_t i = 0; i < a->get_number_of_elements(); ++i) s += double(a->get_data_ptr()[i]) * b->get_data_ptr()[i];
  return T(s);
}

template <class T>
class cuNDArray {
 public:
  using element_type = T;
  cuNDArray() = default;
  explicit cuNDArray(const std::vector<size_t>* d) : dims_(*d), owned_(true) {
    if (cudaMalloc(&data_, bytes()) != cudaSuccess) throw std::runtime_error("cudaMalloc failed");
  }
  explicit cuNDArray(const std::vector<size_t>& d) : cuNDArray(&d) {}
  explicit cuNDArray(const boost::shared_ptr<std::vector<size_t>>& d) : cuNDArray(d.get()) {}
  cuNDArray(const std::vector<size_t>& d, T* ptr) : dims_(d), data_(ptr), owned_(false) {}
  cuNDArray(const cuNDArray&) = delete;
  cuNDArray& operator=(const cuNDArray&) = delete;
  ~cuNDArray() {
    if (owned_ && data_) cudaFree(data_);
  }
  T* get_data_ptr() const { return data_; }
  size_t get_size(size_t i) const { return i < dims_.size() ? dims_[i] : 1; }
  size_t get_number_of_dimensions() const { return dims_.size(); }
  size_t get_number_of_elements() const { return hoCuNDArray<T>::count(dims_); }
  boost::shared_ptr<std::vector<size_t>> get_dimensions() const { return boost::make_shared<std::vector<size_t>>(dims_); }
  size_t bytes() const { return get_number_of_elements() * sizeof(T); }

 private:
  std::vector<size_t> dims_;
  T* data_ = nullptr;
  bool owned_ = false;
};

template <class ARRAY>
class linearOperator {
 public:
  virtual ~linearOperator() = default;
  virtual void mult_M(ARRAY* in, ARRAY* out, bool accumulate = false) = 0;
  virtual void mult_MH(ARRAY* in, ARRAY* out, bool accumulate = false) = 0;
  virtual void set_domain_dimensions(std::vector<size_t>* d) { domain_ = boost::make_shared<std::vector<size_t>>(*d); }
  virtual boost::shared_ptr<std::vector<size_t>> get_domain_dimensions() { return domain_; }
  virtual void set_codomain_dimensions(std::vector<size_t>* d) { codomain_ = boost::make_shared<std::vector<size_t>>(*d); }
  virtual boost::shared_ptr<std::vector<size_t>> get_codomain_dimensions() { return codomain_; }

 protected:
  boost::shared_ptr<std::vector<size_t>> domain_, codomain_;
};

template <class ARRAY>
class subsetOperator : public linearOperator<ARRAY> {
 public:
  explicit subsetOperator(int subsets = 1) : number_of_subsets(subsets) {}
  using linearOperator<ARRAY>::get_codomain_dimensions;
  virtual void mult_M(ARRAY* in, ARRAY* out, int subset, bool accumulate) = 0;
  virtual void mult_MH(ARRAY* in, ARRAY* out, int subset, bool accumulate) = 0;
  virtual void mult_MH_M(ARRAY* in, ARRAY* out, int subset, bool accumulate) = 0;
  virtual boost::shared_ptr<std::vector<size_t>> get_codomain_dimensions(int subset) = 0;
  virtual int get_number_of_subsets() { return number_of_subsets; }
  void mult_M(ARRAY* in, ARRAY* out, bool accumulate = false) override {
    auto p = projection_subsets(out);
    for (int i = 0; i < number_of_subsets; ++i) mult_M(in, p[i].get(), i, accumulate);
  }
  void mult_MH(ARRAY* in, ARRAY* out, bool accumulate = false) override {
    auto p = projection_subsets(in);
    for (int i = 0; i < number_of_subsets; ++i) mult_MH(p[i].get(), out, i, accumulate || i > 0);
  }
  std::vector<boost::shared_ptr<ARRAY>> projection_subsets(ARRAY* projections) {
    std::vector<boost::shared_ptr<ARRAY>> r;
    auto* ptr = projections->get_data_ptr();
    for (int s = 0; s < number_of_subsets; ++s) {
      auto d = *get_codomain_dimensions(s);
      r.push_back(boost::make_shared<ARRAY>(d, ptr));
      ptr += hoCuNDArray<float>::count(d);
    }
    return r;
  }

 protected:
  int number_of_subsets;
};

class CBCT_geometry {
 public:
  void set_SAD(float v) { SAD_ = v; }
  float get_SAD() { return SAD_; }
  void set_SDD(float v) { SDD_ = v; }
  float get_SDD() { return SDD_; }
  void set_FOV(floatd2 v) { FOV_ = v; }
  floatd2 get_FOV() { return FOV_; }
  void set_angles(std::vector<float> a) { angles_ = a; }
  std::vector<float>& get_angles() { return angles_; }
  void set_offsets(std::vector<floatd2>& o) { offsets_ = o; }
  std::vector<floatd2>& get_offsets() { return offsets_; }

 private:
  float SAD_ = 0, SDD_ = 0;
  floatd2 FOV_;
  std::vector<float> angles_;
  std::vector<floatd2> offsets_;
};

class CBCT_acquisition {
 public:
  boost::shared_ptr<CBCT_geometry> get_geometry() { return geometry_; }
  void set_geometry(boost::shared_ptr<CBCT_geometry> g) { geometry_ = g; }
  boost::shared_ptr<hoCuNDArray<float>> get_projections() { return projections_; }
  void set_projections(boost::shared_ptr<hoCuNDArray<float>> p) { projections_ = p; }

 private:
  boost::shared_ptr<CBCT_geometry> geometry_ = boost::make_shared<CBCT_geometry>();
  boost::shared_ptr<hoCuNDArray<float>> projections_;
};

class CBCT_binning {
 public:
  CBCT_binning() = default;
  explicit CBCT_binning(std::vector<std::vector<unsigned int>> b) : bins_(std::move(b)) {}
  std::vector<std::vector<unsigned int>> get_bins() { return bins_; }
  unsigned int get_number_of_bins() { return (unsigned)bins_.size(); }
  std::vector<unsigned int>& get_bin(unsigned b) { return bins_[b]; }

 private:
  std::vector<std::vector<unsigned int>> bins_;
};

}  // namespace Gadgetron
