#pragma once
/**
 * common.h -- exception types of the stereo API (LumenStereo
 * include/stereo/common.h:31-120) mapped from the C ABI's status codes.
 */
#include <stdexcept>
#include <string>

#include "../lumen_sgbm.h"

namespace stereo {

/** A CUDA (or device) failure.  error_code carries the lumen_status. */
class CudaException : public std::runtime_error {
public:
    CudaException(int err, const std::string& msg) : std::runtime_error(msg), error_code(err) {}
    int error_code;
};

/** Invalid input / parameters (empty images, size mismatch, bad range). */
class StereoException : public std::runtime_error {
public:
    explicit StereoException(const std::string& msg) : std::runtime_error(msg) {}
};

class CalibrationException : public StereoException {
public:
    explicit CalibrationException(const std::string& msg)
        : StereoException("Calibration error: " + msg) {}
};

/** Throws the reference's exception type for a non-OK status. */
inline void throwOnError(lumen_status s) {
    if (s == LUMEN_OK) return;
    const std::string msg = lumen_last_error_string();
    if (s == LUMEN_ERR_INVALID_ARGUMENT || s == LUMEN_ERR_RANGE_EXCEEDS_LIMIT ||
        s == LUMEN_ERR_OUT_OF_BUDGET)
        throw StereoException(msg);
    throw CudaException(static_cast<int>(s), msg);
}

inline int divUp(int a, int b) { return (a + b - 1) / b; }

}  // namespace stereo
