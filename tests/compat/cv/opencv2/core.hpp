// Test stand-in for OpenCV's core header: the project-written cv::Mat of the
// reference checker's OpenCV shim (oracle/ref/cvshim), so that the
// reference-interface classes' cv::Mat conversions compile and run here.
#pragma once
#include "../../../../oracle/ref/cvshim/opencv2/opencv.hpp"
