// Complex scalar used by the register DFT codelets and the Q kernels.
#pragma once

namespace bdgfs {

template <typename T>
struct alignas(2 * sizeof(T)) cpx {
    T x, y;
};

}  // namespace bdgfs
