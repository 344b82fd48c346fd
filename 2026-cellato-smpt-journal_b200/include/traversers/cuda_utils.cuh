// CUDA error checking (interface of the reference
// include/traversers/cuda_utils.cuh:11-52): CudaError and the CUCH(...) macro,
// and CELLATO_CHECK for C-ABI status codes.
#ifndef CUCH_HPP
#define CUCH_HPP

#include <cuda_runtime.h>

#include <sstream>
#include <stdexcept>
#include <string>

#include "cellato_b200.h"

class CudaError : public std::exception {
protected:
    std::string mMessage;
    cudaError_t mStatus;

public:
    CudaError(cudaError_t status = cudaSuccess) : mStatus(status) {}
    CudaError(const std::string& msg, cudaError_t status = cudaSuccess) : mMessage(msg), mStatus(status) {}
    const char* what() const noexcept override { return mMessage.c_str(); }
    template <typename T>
    CudaError& operator<<(const T& data) {
        std::stringstream s;
        s << mMessage << data;
        mMessage = s.str();
        return *this;
    }
};

inline void _cuda_check(cudaError_t status, int line, const char* file, const char* what = nullptr) {
    if (status != cudaSuccess)
        throw(CudaError(status) << "CUDA Error (" << status << "): " << cudaGetErrorString(status) << "\n"
                                << "at " << file << ":" << line << ":" << (what ? what : ""));
}
#define CUCH(status) _cuda_check(status, __LINE__, __FILE__, #status)

// C-ABI status -> exception with the library's message
inline void _cellato_check(int status, const char* what) {
    if (status != CELLATO_OK) throw std::runtime_error(std::string(what) + ": " + cellato_last_error());
}
#define CELLATO_CHECK(status) _cellato_check((status), #status)

#endif  // CUCH_HPP
