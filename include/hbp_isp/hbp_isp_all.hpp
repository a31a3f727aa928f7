// All of the reference-interface classes.
#pragma once
#include "CRTrees.hpp"
#include "hbp_isp.hpp"
#include "post_process.hpp"
#include "segment.hpp"
#include "stereo_cost.hpp"
#include "io.hpp"
