// Host runtime pieces shared by the 2-D and 3-D runners behind the C ABI:
// error classes mapped to bhcb status codes, a growable device buffer and the
// table arena that packs an environment's arrays into one upload.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace bhcb {

struct CudaError : std::runtime_error {   // -> BHCB_ERR_CUDA
    using std::runtime_error::runtime_error;
};
struct StateError : std::runtime_error {  // -> BHCB_ERR_STATE
    using std::runtime_error::runtime_error;
};
struct MemError : std::runtime_error {    // -> BHCB_ERR_MEMORY
    using std::runtime_error::runtime_error;
};

#define CK(x)                                                                           \
    do {                                                                                \
        cudaError_t e_ = (x);                                                           \
        if(e_ != cudaSuccess)                                                           \
            throw ::bhcb::CudaError(std::string(#x) + ": " + cudaGetErrorString(e_));   \
    } while(0)

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    void ensure(size_t n)
    {
        if(n <= bytes) return;
        release();
        CK(cudaMalloc(&p, n));
        bytes = n;
    }
    void release()
    {
        if(p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
};

// arrays packed at 256-byte offsets into one host image, uploaded at once;
// each array's space is padded to a multiple of 16 bytes (bulk copies move
// whole 16-byte words)
struct Arena {
    std::vector<uint8_t> bytes;
    template<typename T> size_t put(const std::vector<T> &v)
    {
        size_t off = (bytes.size() + 255) & ~size_t(255);
        bytes.resize(off + std::max<size_t>((v.size() * sizeof(T) + 15) & ~size_t(15), 16));
        if(!v.empty()) std::memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }
};

template<typename T> T *dptr(void *base, size_t off)
{
    return reinterpret_cast<T *>(reinterpret_cast<uint8_t *>(base) + off);
}

// Fortran sequential unformatted records: [int32 n][n bytes][int32 n]
struct RecWriter {
    std::vector<uint8_t> cur;
    std::ofstream &o;
    explicit RecWriter(std::ofstream &o_) : o(o_) {}
    template<typename T> void put(const T &v)
    {
        const uint8_t *p = reinterpret_cast<const uint8_t *>(&v);
        cur.insert(cur.end(), p, p + sizeof(T));
    }
    void put_bytes(const void *p, size_t n)
    {
        const uint8_t *q = reinterpret_cast<const uint8_t *>(p);
        cur.insert(cur.end(), q, q + n);
    }
    void end()
    {
        int32_t n = (int32_t)cur.size();
        o.write((const char *)&n, 4);
        o.write((const char *)cur.data(), cur.size());
        o.write((const char *)&n, 4);
        cur.clear();
    }
};

} // namespace bhcb
