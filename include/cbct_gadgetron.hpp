// cbct_gadgetron.hpp -- drop-in ordered-subset cone-beam operator for gt-tomography.
//
// CBSubsetOperatorB200 is a Gadgetron subsetOperator<cuNDArray<float>> with the
// interface and semantics of gt-tomography's CBSubsetOperator<cuNDArray>
// (xray/CBSubsetOperator.{h,cpp}) and of the cuConebeamProjectionOperator it
// owns per subset (xray/cuConebeamProjectionOperator.{h,cpp}), implemented over
// the C ABI of cbct.h (libcbct.so, hand-written sm_100a kernels).  It drops into
// osMOMSolverD / osSARTSolver unchanged, e.g. in xray/cuCBOS_reconstruct.cpp:
//
//     auto E = boost::make_shared<CBSubsetOperatorB200>(subsets);
//     E->setup(ps, binning, imageDimensions);
//     E->set_domain_dimensions(&is_dims);
//     solver.set_encoding_operator(E);
//
// and offers solve_osmom(), which runs the whole osMOMSolverD loop (no
// regulariser) on the device in one call.  Header-only; link with -lcbct.
// All work runs on the legacy default stream, like the reference.
#pragma once

#include <algorithm>
#include <cmath>
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

class CBSubsetOperatorB200 : public subsetOperator<cuNDArray<float>> {
 public:
  explicit CBSubsetOperatorB200(int subsets = 1) : subsetOperator<cuNDArray<float>>(subsets) {}
  ~CBSubsetOperatorB200() override {
    if (plan_) cbct_plan_destroy(plan_);
  }

  // CBSubsetOperator::setup (CBSubsetOperator.cpp:52-158): round-robin subsets,
  // sorted by bin, and the acquisition's projections and geometry permuted in
  // place into subset-contiguous order.  One bin is supported.
  void setup(boost::shared_ptr<CBCT_acquisition> acq, boost::shared_ptr<CBCT_binning> binning, floatd3 is_dims_in_mm) {
    auto geo = acq->get_geometry();
    std::vector<float> all_angles = geo->get_angles();
    std::vector<floatd2> all_offsets = geo->get_offsets();
    const int P = (int)all_angles.size();
    if (binning->get_number_of_bins() != 1) throw std::runtime_error("Error: CBSubsetOperatorB200: one bin only");
    const float mn = *std::min_element(all_angles.begin(), all_angles.end());
    for (auto& a : all_angles) a -= mn;
    std::vector<int32_t> view_bin(P, -1);
    for (unsigned v : binning->get_bin(0)) view_bin[v] = 0;
    std::vector<int32_t> order(P), sizes(number_of_subsets);
    int32_t n = 0;
    cbct_throw_if(cbct_subset_partition(P, view_bin.data(), number_of_subsets, order.data(), sizes.data(), &n),
                  "CBSubsetOperatorB200::setup");
    order.resize(n);
    // permute the acquisition (CBSubsetOperator.cpp:106-115)
    auto proj = acq->get_projections();
    if (proj) {
      const size_t plane = proj->get_size(0) * proj->get_size(1);
      auto permuted = boost::make_shared<hoCuNDArray<float>>(std::vector<size_t>{proj->get_size(0), proj->get_size(1), (size_t)n});
      for (int i = 0; i < n; ++i)
        std::copy(proj->get_data_ptr() + plane * order[i], proj->get_data_ptr() + plane * (order[i] + 1),
                  permuted->get_data_ptr() + plane * i);
      acq->set_projections(permuted);
      W_ = (int)proj->get_size(0);
      H_ = (int)proj->get_size(1);
    }
    std::vector<float> angles(n);
    std::vector<floatd2> offsets(n);
    for (int i = 0; i < n; ++i) {
      angles[i] = all_angles[order[i]];
      offsets[i] = all_offsets[order[i]];
    }
    geo->set_angles(angles);
    geo->set_offsets(offsets);
    angles_ = angles;
    offsets_.resize(2 * (size_t)n);
    for (int i = 0; i < n; ++i) {
      offsets_[2 * i] = offsets[i][0];
      offsets_[2 * i + 1] = offsets[i][1];
    }
    sizes_ = sizes;
    SAD_ = geo->get_SAD();
    SDD_ = geo->get_SDD();
    fov_ = geo->get_FOV();
    is_dims_in_mm_ = is_dims_in_mm;
    // per-subset offset-correction override (cuConebeamProjectionOperator.cpp:176-181)
    offcorr_.assign(number_of_subsets, 0);
    cbct_geometry g = geometry(1, 1, 1);
    for (int s = 0, f = 0; s < number_of_subsets; f += sizes_[s], ++s)
      if (sizes_[s] > 0) {
        int32_t use = 0;
        cbct_throw_if(cbct_offset_override(&g, offsets_.data() + 2 * f, sizes_[s], &use), "setup");
        offcorr_[s] = use_override_ >= 0 ? use_override_ : use;
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

  boost::shared_ptr<std::vector<size_t>> get_codomain_dimensions(int subset) override {
    return boost::make_shared<std::vector<size_t>>(std::vector<size_t>{(size_t)W_, (size_t)H_, (size_t)sizes_.at(subset)});
  }

  // cuConebeamProjectionOperator::mult_M (.cpp:38-80) of one subset.
  void mult_M(cuNDArray<float>* in, cuNDArray<float>* out, int subset, bool accumulate) override {
    check_arrays(in, out, subset);
    cbct_throw_if(cbct_forward(plan_, subset, CBCT_F32, in->get_data_ptr(), out->get_data_ptr(), accumulate, nullptr),
                  "CBSubsetOperatorB200::mult_M");
  }

  // cuConebeamProjectionOperator::mult_MH (.cpp:82-116): sin^2 offset weight on a copy.
  void mult_MH(cuNDArray<float>* in, cuNDArray<float>* out, int subset, bool accumulate) override {
    check_arrays(out, in, subset);
    cbct_throw_if(cbct_backproject(plan_, subset, in->get_data_ptr(), out->get_data_ptr(), 0, 1, accumulate, nullptr),
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

  // osMOMSolverD<cuNDArray<float>>::solve without regularisers (solvers/osMOMSolverD.h:82-196)
  // as one device-resident call; returns z.
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
    cbct_throw_if(cbct_osmom_solve(plan_, projections->get_data_ptr(), x0 ? x0->get_data_ptr() : nullptr,
                                   z->get_data_ptr(), &prm, nullptr, nullptr),
                  "CBSubsetOperatorB200::solve_osmom");
    return z;
  }

  cbct_plan* plan() { return plan_; }

 private:
  cbct_geometry geometry(int nx, int ny, int nz) const {
    cbct_geometry g{};
    g.SAD = SAD_;
    g.SDD = SDD_;
    g.fov_u = fov_[0];
    g.fov_v = fov_[1];
    g.width = W_;
    g.height = H_;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.lx = is_dims_in_mm_[0];
    g.ly = is_dims_in_mm_[1];
    g.lz = is_dims_in_mm_[2];
    g.samples_per_pixel = 1.5f;  // cuConebeamProjectionOperator.cpp:18
    return g;
  }

  void rebuild() {
    auto d = get_domain_dimensions();
    if (!d || d->size() < 3 || angles_.empty() || W_ == 0) return;
    if (plan_) cbct_plan_destroy(plan_);
    plan_ = nullptr;
    cbct_geometry g = geometry((int)(*d)[0], (int)(*d)[1], (int)(*d)[2]);
    cbct_throw_if(cbct_plan_create(&g, angles_.data(), offsets_.data(), (int)angles_.size(), sizes_.data(),
                                   number_of_subsets, offcorr_.data(), &plan_),
                  "CBSubsetOperatorB200::setup");
  }

  void check_arrays(cuNDArray<float>* vol, cuNDArray<float>* proj, int subset) {
    if (!vol || !proj) throw std::runtime_error("Error: CBSubsetOperatorB200: illegal array pointer provided");
    if (!plan_) throw std::runtime_error("Error: CBSubsetOperatorB200: setup not performed");
    if (subset < 0 || subset >= number_of_subsets) throw std::runtime_error("Error: CBSubsetOperatorB200: subset out of range");
    if (proj->get_number_of_elements() != (size_t)W_ * H_ * sizes_[subset])
      throw std::runtime_error("Error: CBSubsetOperatorB200: inconsistent sizes of input arrays");
  }

  cbct_plan* plan_ = nullptr;
  std::vector<float> angles_, offsets_;
  std::vector<int32_t> sizes_, offcorr_;
  int use_override_ = -1;
  int W_ = 0, H_ = 0;
  float SAD_ = 0, SDD_ = 0;
  floatd2 fov_;
  floatd3 is_dims_in_mm_;
};

}  // namespace Gadgetron
