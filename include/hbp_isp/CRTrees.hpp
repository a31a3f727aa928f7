// CRTrees with the reference's interface (CRTrees.hpp:16-77): connected
// components of a 1-NN successor array on the device (hbp_crtrees_d).
// get_clus leaves the labels already compact (0..n-1 in increasing order of
// the reference's cycle labels); compact_clus_label then returns n.
// nn_d is read only; the cycle mask of show_cycle is not offered.
#pragma once

#include "common.hpp"

namespace hbp_isp
{
class CRTrees
{
  public:
    explicit CRTrees(int size) : m_size(size) {}

    void get_clus(int *nn_d, int *clus_d, int N, int *mask_cycle_d = nullptr)
    {
        if (mask_cycle_d)
            throw std::invalid_argument("CRTrees: the cycle mask is not offered");
        if (N > m_size)
            throw std::invalid_argument("CRTrees: N exceeds the size given at construction");
        detail::check(hbp_crtrees_d(detail::shared_ctx()->h, nn_d, N, clus_d, &m_count, nullptr));
    }

    int compact_clus_label(int *, int) const { return m_count; }

  private:
    int m_size;
    int m_count = 0;
};
} // namespace hbp_isp

#ifndef HBP_ISP_NO_GLOBAL_NAMES
using hbp_isp::CRTrees;
#endif
