// cbct_gadgetron.hpp -- drop-in cone-beam operators for gt-tomography.
//
// Three Gadgetron operators with the interfaces and semantics of gt-tomography's
// cone-beam operators, implemented over the C ABI of cbct.h (libcbct.so,
// hand-written sm_100a kernels):
//
//   cuConebeamProjectionOperatorB200    linearOperator<cuNDArray<float>>
//       xray/cuConebeamProjectionOperator.{h,cpp}: device arrays, bins
//   CBSubsetOperatorB200                subsetOperator<cuNDArray<float>>
//       xray/CBSubsetOperator.{h,cpp} over one cuConebeamProjectionOperator per
//       subset: round-robin subsets, bins, the acquisition permuted in place
//   hoCuConebeamProjectionOperatorB200  linearOperator<hoCuNDArray<float>>
//       xray/hoCuConebeamProjectionOperator.{h,cpp}: host arrays streamed
//       through the device in batches of views, FDK (filtered back-projection)
//
// They drop into the reference's drivers unchanged apart from the class name,
// e.g. xray/cuCBOS_reconstruct.cpp:
//
//     auto E = boost::make_shared<CBSubsetOperatorB200>(subsets);
//     E->setup(ps, binning, imageDimensions);
//     E->set_domain_dimensions(&is_dims);
//     solver.set_encoding_operator(E);
//
// or xray/FDK_reconstruct_3d.cpp:
//
//     boost::shared_ptr<hoCuConebeamProjectionOperatorB200> E(new hoCuConebeamProjectionOperatorB200());
//     E->setup(acquisition, binning, is_dims_in_mm);
//     E->set_use_filtered_backprojection(true);
//     E->mult_MH(&projections, &fdk_3d);
//
// Header-only; link with -lcbct.  Device work runs on the legacy default stream
// and every operator call returns once its work has finished, as the
// reference's do; a kernel that gave up a bounded wait or overflowed its box
// turns into an exception here (cbct_plan_check), as CHECK_FOR_CUDA_ERROR
// turns a CUDA error into one in the reference.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "CBCT_acquisition.h"
#include "CBCT_binning.h"
#include "cbct.h"
#include "cuNDArray.h"
#include "subsetOperator.h"
#include "vector_td.h"

namespace Gadgetron {

inline void cbct_throw_if(cbct_status s, const char* where) {
  if (s != CBCT_OK)
    throw std::runtime_error(std::string("Error: ") + where + ": " + cbct_status_string(s) + ": " + cbct_last_error());
}

namespace cbct_detail {

// The ABI's geometry record from the acquisition's geometry and the image grid.
inline cbct_geometry geometry(CBCT_geometry& geo, int W, int H, int nx, int ny, int nz, floatd3 mm, float spp) {
  cbct_geometry g{};
  g.SAD = geo.get_SAD();
  g.SDD = geo.get_SDD();
  g.fov_u = geo.get_FOV()[0];
  g.fov_v = geo.get_FOV()[1];
  g.width = W;
  g.height = H;
  g.nx = nx;
  g.ny = ny;
  g.nz = nz;
  g.lx = mm[0];
  g.ly = mm[1];
  g.lz = mm[2];
  g.samples_per_pixel = spp;
  return g;
}

// Offset-correction override rule on a set of views (|mean offset_x| > 0.1 FOV_x,
// cuConebeamProjectionOperator.cpp:176-181).
inline bool offset_override(CBCT_geometry& geo, const std::vector<float>& offsets_xy) {
  if (offsets_xy.empty()) return false;
  cbct_geometry g = geometry(geo, 1, 1, 1, 1, 1, floatd3(1.f, 1.f, 1.f), 1.5f);
  int32_t use = 0;
  cbct_throw_if(cbct_offset_override(&g, offsets_xy.data(), (int32_t)(offsets_xy.size() / 2), &use), "setup");
  return use != 0;
}

inline bool short_scan(CBCT_geometry& geo, const std::vector<float>& angles) {
  if (angles.empty()) return false;
  cbct_geometry g = geometry(geo, 1, 1, 1, 1, 1, floatd3(1.f, 1.f, 1.f), 1.5f);
  int32_t ss = 0;
  cbct_throw_if(cbct_is_short_scan(&g, angles.data(), (int32_t)angles.size(), &ss), "setup");
  return ss != 0;
}

inline std::vector<float> flat_offsets(const std::vector<floatd2>& o) {
  std::vector<float> f(2 * o.size());
  for (size_t i = 0; i < o.size(); ++i) {
    f[2 * i] = o[i][0];
    f[2 * i + 1] = o[i][1];
  }
  return f;
}

// Projections permuted into a new view order (the reference's permute_projections,
// cuConebeamProjectionOperator.cpp:225-245, CBSubsetOperator.cpp:190-213).
inline boost::shared_ptr<hoCuNDArray<float>> permute(boost::shared_ptr<hoCuNDArray<float>> proj,
                                                     const std::vector<unsigned>& order) {
  const size_t plane = proj->get_size(0) * proj->get_size(1);
  std::vector<size_t> d{proj->get_size(0), proj->get_size(1), order.size()};
  auto out = boost::make_shared<hoCuNDArray<float>>(d);
  for (size_t i = 0; i < order.size(); ++i)
    std::memcpy(out->get_data_ptr() + plane * i, proj->get_data_ptr() + plane * order[i], plane * sizeof(float));
  return out;
}

// A plan that follows the operator's arrays: made (or remade) on the first call
// with a given detector and image grid, since the reference takes both from the
// arrays it is handed.
struct PlanHolder {
  cbct_plan* plan = nullptr;
  std::vector<int> key;
  ~PlanHolder() { reset(); }
  void reset() {
    if (plan) cbct_plan_destroy(plan);
    plan = nullptr;
    key.clear();
  }
};

}  // namespace cbct_detail

// ----------------------------------------------------------------------------
// cuConebeamProjectionOperatorB200 (xray/cuConebeamProjectionOperator.h:21-53)
// ----------------------------------------------------------------------------
// Images are (nx, ny, nz) or (nx, ny, nz, bins); projections hold the bins'
// views in bin order (the order setup leaves the acquisition's projections in).
// Differences from the reference, on purpose: use_offset_correction starts
// false (the reference leaves it uninitialised unless the override fires,
// .cpp:15-21), and without a binning every view forms one bin (the reference
// sizes its default bin from a member that is still empty, .cpp:183-187).
class cuConebeamProjectionOperatorB200 : public linearOperator<cuNDArray<float>> {
 public:
  cuConebeamProjectionOperatorB200() = default;

  // cuConebeamProjectionOperator::setup (.cpp:148-206).
  void setup(boost::shared_ptr<CBCT_acquisition> acquisition, boost::shared_ptr<CBCT_binning> binning,
             floatd3 is_dims_in_mm, bool transform_angles = true) {
    binning_ = binning;
    setup(acquisition, is_dims_in_mm, transform_angles);
  }

  void setup(boost::shared_ptr<CBCT_acquisition> acquisition, floatd3 is_dims_in_mm, bool transform_angles = true) {
    acquisition_ = acquisition;
    is_dims_in_mm_ = is_dims_in_mm;
    auto geo = acquisition->get_geometry();
    std::vector<float>& all_angles = geo->get_angles();
    if (transform_angles && !all_angles.empty()) {
      const float mn = *std::min_element(all_angles.begin(), all_angles.end());
      for (auto& a : all_angles) a -= mn;
    }
    const std::vector<float> all_off = cbct_detail::flat_offsets(geo->get_offsets());
    short_scan_ = cbct_detail::short_scan(*geo, all_angles);
    if (allow_offset_correction_override_ && cbct_detail::offset_override(*geo, all_off)) use_offset_correction_ = true;
    if (!binning_) {
      std::vector<unsigned> all(all_angles.size());
      std::iota(all.begin(), all.end(), 0u);
      binning_ = boost::make_shared<CBCT_binning>(std::vector<std::vector<unsigned>>(1, all));
    }
    order_.clear();
    view_bin_.clear();
    angles_.clear();
    offsets_.clear();
    for (unsigned b = 0; b < binning_->get_number_of_bins(); ++b)
      for (unsigned v : binning_->get_bin(b)) {
        if (v >= all_angles.size()) throw std::runtime_error("Error: cuConebeamProjectionOperatorB200: illegal view index in bin");
        order_.push_back(v);
        view_bin_.push_back((int32_t)b);
        angles_.push_back(all_angles[v]);
        offsets_.push_back(all_off[2 * v]);
        offsets_.push_back(all_off[2 * v + 1]);
      }
    auto proj = acquisition->get_projections();
    if (proj) acquisition->set_projections(cbct_detail::permute(proj, order_));
    preprocessed_ = true;
    holder_.reset();
  }

  void mult_M(cuNDArray<float>* in, cuNDArray<float>* out, bool accumulate = false) override {
    cbct_plan* p = plan_for(in, out, "mult_M");
    cbct_throw_if(cbct_forward(p, -1, CBCT_F32, in->get_data_ptr(), out->get_data_ptr(), accumulate ? 1 : 0, nullptr),
                  "cuConebeamProjectionOperatorB200::mult_M");
    cbct_throw_if(cbct_plan_check(p, nullptr), "cuConebeamProjectionOperatorB200::mult_M");
  }

  // mult_MH (.cpp:82-116): the sin^2 offset weight on a copy of the input when
  // offset correction is on, and the mask applied to the whole output after.
  void mult_MH(cuNDArray<float>* in, cuNDArray<float>* out, bool accumulate = false) override {
    cbct_plan* p = plan_for(out, in, "mult_MH");
    cbct_throw_if(cbct_backproject(p, -1, in->get_data_ptr(), out->get_data_ptr(), 0, 1, accumulate ? 1 : 0, nullptr),
                  "cuConebeamProjectionOperatorB200::mult_MH");
    if (mask_)
      cbct_throw_if(cbct_apply_mask(out->get_data_ptr(), reinterpret_cast<const uint8_t*>(mask_->get_data_ptr()),
                                    out->get_number_of_elements(), nullptr),
                    "cuConebeamProjectionOperatorB200::mult_MH");
    cbct_throw_if(cbct_plan_check(p, nullptr), "cuConebeamProjectionOperatorB200::mult_MH");
  }

  // offset_correct (.cpp:22-31): the sqrt (sin) weight in place on every view.
  void offset_correct(cuNDArray<float>* projections) {
    if (!preprocessed_) throw std::runtime_error("Error: cuConebeamProjectionOperatorB200::offset_correct: setup not performed");
    cbct_plan* p = plan_for_projections(projections, "offset_correct");
    cbct_throw_if(cbct_offset_correct(p, -1, projections->get_data_ptr(), 1, nullptr), "offset_correct");
  }

  // calculate_mask (.cpp:118-147): the space carver, one per bin.
  boost::shared_ptr<cuNDArray<bool>> calculate_mask(cuNDArray<float>* projections, float limit) {
    auto dims = get_domain_dimensions();
    if (!dims) throw std::runtime_error("Error: cuConebeamProjectionOperatorB200::calculate_mask: no domain dimensions");
    auto mask = boost::make_shared<cuNDArray<bool>>(dims.get());
    const size_t nvox = (*dims)[0] * (*dims)[1] * (*dims)[2];
    const size_t plane = projections->get_size(0) * projections->get_size(1);
    size_t first = 0;
    for (unsigned b = 0; b < binning_->get_number_of_bins(); ++b) {
      const size_t n = binning_->get_bin(b).size();
      uint8_t* m = reinterpret_cast<uint8_t*>(mask->get_data_ptr()) + nvox * b;
      if (n == 0) {
        cudaMemset(m, 1, nvox);
        continue;
      }
      auto geo = acquisition_->get_geometry();
      cbct_geometry g = cbct_detail::geometry(*geo, (int)projections->get_size(0), (int)projections->get_size(1),
                                              (int)(*dims)[0], (int)(*dims)[1], (int)(*dims)[2], is_dims_in_mm_,
                                              samples_per_pixel_);
      cbct_plan* bp = nullptr;
      cbct_throw_if(cbct_plan_create(&g, angles_.data() + first, offsets_.data() + 2 * first, (int32_t)n, nullptr, 1,
                                     nullptr, &bp),
                    "calculate_mask");
      const cbct_status st = cbct_spacecarver(bp, -1, projections->get_data_ptr() + plane * first, limit, m, 0, nullptr);
      cbct_plan_destroy(bp);
      cbct_throw_if(st, "calculate_mask");
      first += n;
    }
    cbct_throw_if(cudaDeviceSynchronize() == cudaSuccess ? CBCT_OK : CBCT_ERR_CUDA, "calculate_mask");
    return mask;
  }

  bool get_use_offset_correction() { return use_offset_correction_; }
  void set_use_offset_correction(bool use) {
    use_offset_correction_ = use;
    allow_offset_correction_override_ = false;
    holder_.reset();
  }
  void set_mask(boost::shared_ptr<cuNDArray<bool>> m) { mask_ = m; }

 protected:
  // The plan for an image of `img`'s grid and projections of `proj`'s detector.
  cbct_plan* plan_for(cuNDArray<float>* img, cuNDArray<float>* proj, const char* what) {
    if (!img || !proj) throw std::runtime_error(std::string("Error: cuConebeamProjectionOperatorB200::") + what +
                                                ": illegal array pointer provided");
    if (!preprocessed_) throw std::runtime_error(std::string("Error: cuConebeamProjectionOperatorB200::") + what +
                                                 ": setup not performed");
    const size_t bins = img->get_number_of_dimensions() == 4 ? img->get_size(3) : 1;
    if (bins != binning_->get_number_of_bins() || proj->get_size(2) != angles_.size())
      throw std::runtime_error(std::string("Error: cuConebeamProjectionOperatorB200::") + what +
                               ": inconsistent sizes of input arrays/vectors");
    return plan((int)proj->get_size(0), (int)proj->get_size(1), (int)img->get_size(0), (int)img->get_size(1),
                (int)img->get_size(2));
  }

  cbct_plan* plan_for_projections(cuNDArray<float>* proj, const char* what) {
    auto d = get_domain_dimensions();
    if (!d || d->size() < 3)
      throw std::runtime_error(std::string("Error: cuConebeamProjectionOperatorB200::") + what + ": no domain dimensions");
    return plan((int)proj->get_size(0), (int)proj->get_size(1), (int)(*d)[0], (int)(*d)[1], (int)(*d)[2]);
  }

  cbct_plan* plan(int W, int H, int nx, int ny, int nz) {
    std::vector<int> key{W, H, nx, ny, nz};
    if (holder_.plan && holder_.key == key) return holder_.plan;
    holder_.reset();
    cbct_geometry g = cbct_detail::geometry(*acquisition_->get_geometry(), W, H, nx, ny, nz, is_dims_in_mm_,
                                            samples_per_pixel_);
    const int32_t oc = use_offset_correction_ ? 1 : 0;
    cbct_throw_if(cbct_plan_create(&g, angles_.data(), offsets_.data(), (int32_t)angles_.size(), nullptr, 1, &oc,
                                   &holder_.plan),
                  "cuConebeamProjectionOperatorB200::setup");
    if (binning_->get_number_of_bins() > 1)
      cbct_throw_if(cbct_plan_set_bins(holder_.plan, (int32_t)binning_->get_number_of_bins(), view_bin_.data()),
                    "cuConebeamProjectionOperatorB200::setup");
    holder_.key = key;
    return holder_.plan;
  }

  boost::shared_ptr<CBCT_acquisition> acquisition_;
  boost::shared_ptr<CBCT_binning> binning_;
  boost::shared_ptr<cuNDArray<bool>> mask_;
  std::vector<unsigned> order_;
  std::vector<int32_t> view_bin_;
  std::vector<float> angles_, offsets_;   // the bins' views in bin order
  floatd3 is_dims_in_mm_;
  float samples_per_pixel_ = 1.5f;       // .cpp:18
  bool preprocessed_ = false;
  bool short_scan_ = false;
  bool use_offset_correction_ = false;
  bool allow_offset_correction_override_ = true;
  cbct_detail::PlanHolder holder_;
};

// ----------------------------------------------------------------------------
// CBSubsetOperatorB200 (xray/CBSubsetOperator.h:30-72, .cpp:19-215)
// ----------------------------------------------------------------------------
class CBSubsetOperatorB200 : public subsetOperator<cuNDArray<float>> {
 public:
  explicit CBSubsetOperatorB200(int subsets = 1) : subsetOperator<cuNDArray<float>>(subsets) {}
  ~CBSubsetOperatorB200() override {
    if (plan_) cbct_plan_destroy(plan_);
  }

  // CBSubsetOperator::setup (CBSubsetOperator.cpp:52-158): views in the bins
  // dealt round-robin to the subsets, each subset sorted by bin, the
  // acquisition's projections and geometry permuted in place into
  // subset-contiguous order, per-subset offset-correction override.  Images
  // hold one volume per bin (nx, ny, nz[, bins]).
  void setup(boost::shared_ptr<CBCT_acquisition> acq, boost::shared_ptr<CBCT_binning> binning, floatd3 is_dims_in_mm) {
    auto geo = acq->get_geometry();
    std::vector<float> all_angles = geo->get_angles();
    std::vector<floatd2> all_offsets = geo->get_offsets();
    const int P = (int)all_angles.size();
    const float mn = *std::min_element(all_angles.begin(), all_angles.end());
    for (auto& a : all_angles) a -= mn;
    n_bins_ = (int)binning->get_number_of_bins();
    std::vector<int32_t> view_bin(P, -1);
    for (int b = 0; b < n_bins_; ++b)
      for (unsigned v : binning->get_bin(b)) {
        if ((int)v >= P) throw std::runtime_error("Error: CBSubsetOperatorB200::setup: illegal view index in bin");
        view_bin[v] = b;
      }
    std::vector<int32_t> order(P), sizes(number_of_subsets);
    int32_t n = 0;
    cbct_throw_if(cbct_subset_partition(P, view_bin.data(), number_of_subsets, order.data(), sizes.data(), &n),
                  "CBSubsetOperatorB200::setup");
    order.resize(n);
    // permute the acquisition (CBSubsetOperator.cpp:100-115)
    auto proj = acq->get_projections();
    if (proj) {
      W_ = (int)proj->get_size(0);
      H_ = (int)proj->get_size(1);
      acq->set_projections(cbct_detail::permute(proj, std::vector<unsigned>(order.begin(), order.end())));
    }
    std::vector<float> angles(n);
    std::vector<floatd2> offsets(n);
    plan_bin_.assign(n, 0);
    for (int i = 0; i < n; ++i) {
      angles[i] = all_angles[order[i]];
      offsets[i] = all_offsets[order[i]];
      plan_bin_[i] = view_bin[order[i]];
    }
    geo->set_angles(angles);
    geo->set_offsets(offsets);
    angles_ = angles;
    offsets_ = cbct_detail::flat_offsets(offsets);
    sizes_ = sizes;
    geo_ = *geo;
    is_dims_in_mm_ = is_dims_in_mm;
    // per-subset offset-correction override (each subset's own
    // cuConebeamProjectionOperator::setup, .cpp:176-181)
    offcorr_.assign(number_of_subsets, 0);
    for (int s = 0, f = 0; s < number_of_subsets; f += sizes_[s], ++s) {
      std::vector<float> so(offsets_.begin() + 2 * f, offsets_.begin() + 2 * (f + sizes_[s]));
      offcorr_[s] = use_override_ >= 0 ? use_override_ : (cbct_detail::offset_override(geo_, so) ? 1 : 0);
    }
    rebuild();
  }

  void setup(boost::shared_ptr<CBCT_acquisition> acq, floatd3 is_dims_in_mm) {
    std::vector<unsigned int> all(acq->get_geometry()->get_angles().size());
    std::iota(all.begin(), all.end(), 0u);
    setup(acq, boost::make_shared<CBCT_binning>(std::vector<std::vector<unsigned int>>(1, all)), is_dims_in_mm);
  }

  void set_domain_dimensions(std::vector<size_t>* dims) override {
    subsetOperator<cuNDArray<float>>::set_domain_dimensions(dims);
    rebuild();
  }

  void set_use_offset_correction(bool use) {
    use_override_ = use ? 1 : 0;
    std::fill(offcorr_.begin(), offcorr_.end(), use_override_);
    rebuild();
  }

  bool get_use_offset_correction(int subset) { return offcorr_.at(subset) != 0; }

  boost::shared_ptr<std::vector<size_t>> get_codomain_dimensions(int subset) override {
    return boost::make_shared<std::vector<size_t>>(std::vector<size_t>{(size_t)W_, (size_t)H_, (size_t)sizes_.at(subset)});
  }

  // cuConebeamProjectionOperator::mult_M (.cpp:38-80) of one subset: each bin's
  // views project that bin's volume.
  void mult_M(cuNDArray<float>* in, cuNDArray<float>* out, int subset, bool accumulate) override {
    check_arrays(in, out, subset);
    cbct_throw_if(cbct_forward(plan_, subset, CBCT_F32, in->get_data_ptr(), out->get_data_ptr(), accumulate, nullptr),
                  "CBSubsetOperatorB200::mult_M");
  }

  // cuConebeamProjectionOperator::mult_MH (.cpp:82-116): sin^2 offset weight on
  // a copy, each bin's volume from its own views, the mask on the output.
  void mult_MH(cuNDArray<float>* in, cuNDArray<float>* out, int subset, bool accumulate) override {
    check_arrays(out, in, subset);
    cbct_throw_if(cbct_backproject(plan_, subset, in->get_data_ptr(), out->get_data_ptr(), 0, 1, accumulate, nullptr),
                  "CBSubsetOperatorB200::mult_MH");
    if (mask_)
      cbct_throw_if(cbct_apply_mask(out->get_data_ptr(), reinterpret_cast<const uint8_t*>(mask_->get_data_ptr()),
                                    out->get_number_of_elements(), nullptr),
                    "CBSubsetOperatorB200::mult_MH");
  }

  void mult_MH_M(cuNDArray<float>* in, cuNDArray<float>* out, int subset, bool accumulate) override {
    auto d = *get_codomain_dimensions(subset);
    cuNDArray<float> tmp(&d);
    mult_M(in, &tmp, subset, false);
    mult_MH(&tmp, out, subset, accumulate);
  }

  using subsetOperator<cuNDArray<float>>::mult_M;
  using subsetOperator<cuNDArray<float>>::mult_MH;

  // CBSubsetOperator::offset_correct (.cpp:44-50): sqrt weight where enabled.
  void offset_correct(cuNDArray<float>* projections) {
    auto sets = projection_subsets(projections);
    for (int s = 0; s < number_of_subsets; ++s)
      if (offcorr_[s]) cbct_throw_if(cbct_offset_correct(plan_, s, sets[s]->get_data_ptr(), 1, nullptr), "offset_correct");
  }

  // CBSubsetOperator::calculate_mask (.cpp:168-181): the AND of every subset's
  // space-carved mask (one bin).
  boost::shared_ptr<cuNDArray<bool>> calculate_mask(boost::shared_ptr<cuNDArray<float>> projections, float limit) {
    if (n_bins_ > 1) throw std::runtime_error("Error: CBSubsetOperatorB200::calculate_mask: one bin only");
    auto dims = get_domain_dimensions();
    auto mask = boost::make_shared<cuNDArray<bool>>(dims.get());
    cudaMemset(mask->get_data_ptr(), 1, mask->get_number_of_elements());
    auto sets = projection_subsets(projections.get());
    for (int s = 0; s < number_of_subsets; ++s)
      cbct_throw_if(cbct_spacecarver(plan_, s, sets[s]->get_data_ptr(), limit,
                                     reinterpret_cast<uint8_t*>(mask->get_data_ptr()), 1, nullptr),
                    "calculate_mask");
    return mask;
  }

  void set_mask(boost::shared_ptr<cuNDArray<bool>> m) { mask_ = m; }

  // osMOMSolverD<cuNDArray<float>>::solve without regularisers (solvers/osMOMSolverD.h:82-196)
  // as one device-resident call; returns z (one volume per bin).
  boost::shared_ptr<cuNDArray<float>> solve_osmom(cuNDArray<float>* projections, int iterations, bool non_negativity,
                                                  float beta = 1.f, float gamma = 0.f, cuNDArray<float>* x0 = nullptr) {
    auto dims = *get_domain_dimensions();
    auto z = boost::make_shared<cuNDArray<float>>(&dims);
    cbct_solver_params prm{};
    prm.iterations = iterations;
    prm.beta = beta;
    prm.gamma = gamma;
    prm.non_negativity = non_negativity ? 1 : 0;
    prm.use_graph = 0;
    prm.storage = CBCT_F32;
    prm.refine_every = 0;
    prm.proj_storage = CBCT_F32;
    prm.tau = 1e-3f;
    prm.reg_steps = 1;
    if (mask_ && n_bins_ > 1)
      throw std::runtime_error("Error: CBSubsetOperatorB200::solve_osmom: a mask with several bins is not supported");
    if (mask_) cbct_throw_if(cbct_plan_set_mask(plan_, reinterpret_cast<const uint8_t*>(mask_->get_data_ptr())),
                             "CBSubsetOperatorB200::solve_osmom");
    const cbct_status st = cbct_osmom_solve(plan_, projections->get_data_ptr(), x0 ? x0->get_data_ptr() : nullptr,
                                            z->get_data_ptr(), &prm, nullptr, nullptr);
    if (mask_) cbct_plan_set_mask(plan_, nullptr);
    cbct_throw_if(st, "CBSubsetOperatorB200::solve_osmom");
    return z;
  }

  cbct_plan* plan() { return plan_; }

 private:
  void rebuild() {
    auto d = get_domain_dimensions();
    if (!d || d->size() < 3 || angles_.empty() || W_ == 0) return;
    if (n_bins_ > 1 && (d->size() < 4 || (int)(*d)[3] != n_bins_))
      throw std::runtime_error("Error: CBSubsetOperatorB200: a binned setup needs domain dimensions (nx, ny, nz, bins)");
    if (plan_) cbct_plan_destroy(plan_);
    plan_ = nullptr;
    cbct_geometry g = cbct_detail::geometry(geo_, W_, H_, (int)(*d)[0], (int)(*d)[1], (int)(*d)[2], is_dims_in_mm_, 1.5f);
    cbct_throw_if(cbct_plan_create(&g, angles_.data(), offsets_.data(), (int)angles_.size(), sizes_.data(),
                                   number_of_subsets, offcorr_.data(), &plan_),
                  "CBSubsetOperatorB200::setup");
    if (n_bins_ > 1)
      cbct_throw_if(cbct_plan_set_bins(plan_, n_bins_, plan_bin_.data()), "CBSubsetOperatorB200::setup");
  }

  void check_arrays(cuNDArray<float>* vol, cuNDArray<float>* proj, int subset) {
    if (!vol || !proj) throw std::runtime_error("Error: CBSubsetOperatorB200: illegal array pointer provided");
    if (!plan_) throw std::runtime_error("Error: CBSubsetOperatorB200: setup not performed");
    if (subset < 0 || subset >= number_of_subsets) throw std::runtime_error("Error: CBSubsetOperatorB200: subset out of range");
    if (proj->get_number_of_elements() != (size_t)W_ * H_ * sizes_[subset])
      throw std::runtime_error("Error: CBSubsetOperatorB200: inconsistent sizes of input arrays");
  }

  cbct_plan* plan_ = nullptr;
  CBCT_geometry geo_;
  boost::shared_ptr<cuNDArray<bool>> mask_;
  std::vector<float> angles_, offsets_;
  std::vector<int32_t> sizes_, offcorr_, plan_bin_;
  int n_bins_ = 1;
  int use_override_ = -1;
  int W_ = 0, H_ = 0;
  floatd3 is_dims_in_mm_;
};

// ----------------------------------------------------------------------------
// hoCuConebeamProjectionOperatorB200 (xray/hoCuConebeamProjectionOperator.h:17-156,
// .cpp:104-265)
// ----------------------------------------------------------------------------
// Host images (nx, ny, nz[, bins]) and projections (W, H, P) in acquisition
// order.  Each bin's volume stays on the device while its views stream
// through two device buffers of projections_per_batch views (default 20), as
// the reference's host-array projectors do (conebeam_projection.cu:640-819,
// :1300-1649).  With filtered back-projection on, mult_MH is FDK: cosine
// weight, [Parker weight on a short scan], the frequency filter (the default
// filter of compute_default_frequency_filter unless one is set), [sin^2 offset
// weight], 1/U^2-weighted back-projection, and 2/P per bin.
class hoCuConebeamProjectionOperatorB200 : public linearOperator<hoCuNDArray<float>> {
 public:
  hoCuConebeamProjectionOperatorB200() = default;

  void setup(boost::shared_ptr<CBCT_acquisition> acquisition, floatd3 is_dims_in_mm, bool transform_angles = true) {
    acquisition_ = acquisition;
    is_dims_in_mm_ = is_dims_in_mm;
    auto geo = acquisition->get_geometry();
    std::vector<float>& angles = geo->get_angles();
    if (transform_angles && !angles.empty()) {
      const float mn = *std::min_element(angles.begin(), angles.end());
      for (auto& a : angles) a -= mn;
    }
    short_scan_ = cbct_detail::short_scan(*geo, angles);
    if (allow_offset_correction_override_ && cbct_detail::offset_override(*geo, cbct_detail::flat_offsets(geo->get_offsets())))
      use_offset_correction_ = true;
    preprocessed_ = true;
    std::vector<unsigned> bins(angles.size());
    std::iota(bins.begin(), bins.end(), 0u);
    binning_ = boost::make_shared<CBCT_binning>(std::vector<std::vector<unsigned>>(1, bins));
    holder_.reset();
  }

  void setup(boost::shared_ptr<CBCT_acquisition> acquisition, boost::shared_ptr<CBCT_binning> binning,
             floatd3 is_dims_in_mm, bool transform_angles = true) {
    setup(acquisition, is_dims_in_mm, transform_angles);
    binning_ = binning;
  }

  // mult_M (.cpp:104-176): [the sqrt offset weight when offset correction is on
  // and FBP is off], accumulate through a temporary.
  void mult_M(hoCuNDArray<float>* image, hoCuNDArray<float>* projections, bool accumulate = false) override {
    check(image, projections, "mult_M");
    cbct_plan* p = plan_for((int)projections->get_size(0), (int)projections->get_size(1), image);
    hoCuNDArray<float>* target = projections;
    hoCuNDArray<float> tmp;
    if (accumulate) {
      tmp = hoCuNDArray<float>(projections->get_dimensions());
      target = &tmp;
    }
    const size_t nvox = image->get_size(0) * image->get_size(1) * image->get_size(2);
    const int32_t offset = (use_offset_correction_ && !use_fbp_) ? 1 : 0;
    for (size_t b = 0; b < batches_.size(); ++b) {
      if (batches_[b].views == 0) continue;
      cbct_throw_if(cbct_host_forward(p, batches_[b].first, batches_[b].count, image->get_data_ptr() + nvox * b,
                                      target->get_data_ptr(), view_index_.data(), offset, nullptr),
                    "hoCuConebeamProjectionOperatorB200::mult_M");
    }
    if (accumulate)
      for (size_t i = 0; i < projections->get_number_of_elements(); ++i)
        projections->get_data_ptr()[i] += tmp.get_data_ptr()[i];
  }

  // mult_MH (.cpp:178-265): FDK with FBP on, else the plain back-projection
  // with the sqrt offset weight when offset correction is on.
  void mult_MH(hoCuNDArray<float>* projections, hoCuNDArray<float>* image, bool accumulate = false) override {
    check(image, projections, "mult_MH");
    cbct_plan* p = plan_for((int)projections->get_size(0), (int)projections->get_size(1), image);
    const size_t nvox = image->get_size(0) * image->get_size(1) * image->get_size(2);
    const float* filt = filter_.empty() ? nullptr : filter_.data();
    if (filt && filter_.size() != projections->get_size(0) + 1)
      throw std::runtime_error("Error: hoCuConebeamProjectionOperatorB200::mult_MH: the frequency filter needs W+1 bins");
    for (size_t b = 0; b < batches_.size(); ++b) {
      float* img = image->get_data_ptr() + nvox * b;
      cbct_status st;
      if (use_fbp_) {
        const uint32_t flags = (short_scan_ ? CBCT_FDK_PARKER : 0u) | (use_offset_correction_ ? CBCT_FDK_OFFSET : 0u);
        const float scale = batches_[b].views ? 2.f / float(batches_[b].views) : 1.f;
        st = cbct_host_backproject(p, batches_[b].first, batches_[b].count, projections->get_data_ptr(), img,
                                   view_index_.data(), 1, filt, flags, 0, scale, accumulate ? 1 : 0, nullptr);
      } else {
        st = cbct_host_backproject(p, batches_[b].first, batches_[b].count, projections->get_data_ptr(), img,
                                   view_index_.data(), 0, nullptr, 0, use_offset_correction_ ? 1 : 0, 1.f,
                                   accumulate ? 1 : 0, nullptr);
      }
      cbct_throw_if(st, "hoCuConebeamProjectionOperatorB200::mult_MH");
    }
  }

  inline void set_use_filtered_backprojection(bool use_fbp) { use_fbp_ = use_fbp; }
  inline void set_use_offset_correction(bool use_correction) {
    use_offset_correction_ = use_correction;
    allow_offset_correction_override_ = false;
  }
  inline bool get_use_offset_correction() { return use_offset_correction_; }
  inline void set_num_projections_per_batch(unsigned int n) {
    if (n == 0) throw std::runtime_error("Error: hoCuConebeamProjectionOperatorB200: projections per batch must be >= 1");
    projections_per_batch_ = n;
    holder_.reset();
  }
  inline void set_num_samples_per_pixel(float spp) {
    samples_per_pixel_ = spp;
    holder_.reset();
  }
  // set_frequency_filter (.h:117-119): W+1 device floats, used as given (no normalisation).
  inline void set_frequency_filter(boost::shared_ptr<cuNDArray<float>> weights) {
    filter_.resize(weights->get_number_of_elements());
    if (cudaMemcpy(filter_.data(), weights->get_data_ptr(), filter_.size() * sizeof(float), cudaMemcpyDeviceToHost) !=
        cudaSuccess)
      throw std::runtime_error("Error: hoCuConebeamProjectionOperatorB200::set_frequency_filter: copy failed");
  }
  void set_acquisition(boost::shared_ptr<CBCT_acquisition> acquisition) {
    acquisition_ = acquisition;
    holder_.reset();
  }
  boost::shared_ptr<CBCT_acquisition> get_acquisition() { return acquisition_; }
  void set_binning(boost::shared_ptr<CBCT_binning> binning) {
    binning_ = binning;
    holder_.reset();
  }
  boost::shared_ptr<CBCT_binning> get_binning() { return binning_; }

 protected:
  struct Batches {
    int first = 0, count = 0, views = 0;   // plan subsets [first, first + count), the bin's view count
  };

  void check(hoCuNDArray<float>* image, hoCuNDArray<float>* projections, const char* what) {
    const std::string w = std::string("Error: hoCuConebeamProjectionOperatorB200::") + what;
    if (!image || !projections) throw std::runtime_error(w + ": illegal array pointer provided");
    if (image->get_number_of_dimensions() != 3 && image->get_number_of_dimensions() != 4)
      throw std::runtime_error(w + ": image array must be four or three -dimensional");
    if (projections->get_number_of_dimensions() != 3)
      throw std::runtime_error(w + ": projections array must be three-dimensional");
    if (!preprocessed_) throw std::runtime_error(w + ": setup not performed");
    if (!binning_) throw std::runtime_error(w + ": binning not provided");
    auto geo = acquisition_->get_geometry();
    if (projections->get_size(2) != geo->get_angles().size() || projections->get_size(2) != geo->get_offsets().size())
      throw std::runtime_error(w + ": inconsistent sizes of input arrays/vectors");
    const size_t bins = image->get_number_of_dimensions() == 4 ? image->get_size(3) : 1;
    if (bins < binning_->get_number_of_bins()) throw std::runtime_error(w + ": image holds fewer volumes than bins");
  }

  // The plan whose views are the bins' views in bin order, cut into batches
  // of projections_per_batch views (the plan's subsets).
  cbct_plan* plan_for(int W, int H, hoCuNDArray<float>* image) {
    std::vector<int> key{W, H, (int)image->get_size(0), (int)image->get_size(1), (int)image->get_size(2)};
    if (holder_.plan && holder_.key == key) return holder_.plan;
    holder_.reset();
    auto geo = acquisition_->get_geometry();
    const std::vector<float>& angles = geo->get_angles();
    const std::vector<float> off = cbct_detail::flat_offsets(geo->get_offsets());
    std::vector<float> a, o;
    std::vector<int32_t> sizes;
    view_index_.clear();
    batches_.clear();
    const int B = (int)projections_per_batch_;
    for (unsigned b = 0; b < binning_->get_number_of_bins(); ++b) {
      const std::vector<unsigned>& views = binning_->get_bin(b);
      Batches bt;
      bt.first = (int)sizes.size();
      bt.views = (int)views.size();
      for (size_t k = 0; k < views.size(); k += B) sizes.push_back((int32_t)std::min<size_t>(B, views.size() - k));
      bt.count = (int)sizes.size() - bt.first;
      for (unsigned v : views) {
        if (v >= angles.size()) throw std::runtime_error("Error: hoCuConebeamProjectionOperatorB200: illegal index in bin");
        view_index_.push_back((int32_t)v);
        a.push_back(angles[v]);
        o.push_back(off[2 * v]);
        o.push_back(off[2 * v + 1]);
      }
      batches_.push_back(bt);
    }
    if (a.empty()) throw std::runtime_error("Error: hoCuConebeamProjectionOperatorB200: the bins hold no views");
    cbct_geometry g = cbct_detail::geometry(*geo, W, H, key[2], key[3], key[4], is_dims_in_mm_, samples_per_pixel_);
    cbct_throw_if(cbct_plan_create(&g, a.data(), o.data(), (int32_t)a.size(), sizes.data(), (int32_t)sizes.size(),
                                   nullptr, &holder_.plan),
                  "hoCuConebeamProjectionOperatorB200::setup");
    holder_.key = key;
    return holder_.plan;
  }

  boost::shared_ptr<CBCT_acquisition> acquisition_;
  boost::shared_ptr<CBCT_binning> binning_;
  floatd3 is_dims_in_mm_;
  float samples_per_pixel_ = 1.5f;          // .h:22
  unsigned int projections_per_batch_ = 20; // .h:23
  bool use_fbp_ = false;
  bool preprocessed_ = false;
  bool short_scan_ = false;
  bool use_offset_correction_ = false;
  bool allow_offset_correction_override_ = true;
  std::vector<float> filter_;
  std::vector<int32_t> view_index_;
  std::vector<Batches> batches_;
  cbct_detail::PlanHolder holder_;
};

}  // namespace Gadgetron
