// drive.cuh -- the pulse envelope shared by every kernel that applies a drive.
#pragma once

namespace cmd {

// Drive envelope of lattice_md.cpp:45-56: a * exp(-(x/(2w))^2) * cos(freq x).
__device__ __forceinline__ double drive_factor(double amp, double x, double width, double freq) {
    const double u = x / (2.0 * width);
    return amp * exp(-(u * u)) * cos(freq * x);
}

}  // namespace cmd
