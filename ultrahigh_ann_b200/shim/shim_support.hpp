// Support for the reference-side binding: the C++ classes of the reference's
// CUDA API (include/ultrahigh_ann/...) implemented over the engine's C ABI
// (include/uha_b200.h). These sources compile inside the reference project, in
// place of its CUDA translation units; they include the reference's headers.
#pragma once

#include "uha_b200.h"

#include <cstdint>
#include <random>
#include <sstream>
#include <stdexcept>
#include <string>

namespace ultrahigh_ann::engine {

// Rethrows a failed C-ABI status as the reference's exception type.
inline void check(uha_status status)
{
    if (status == UHA_OK) {
        return;
    }
    const std::string message = uha_last_error();
    switch (status) {
    case UHA_INVALID_ARGUMENT:
        throw std::invalid_argument(message);
    case UHA_LENGTH_ERROR:
        throw std::length_error(message);
    case UHA_OVERFLOW_ERROR:
        throw std::overflow_error(message);
    case UHA_OUT_OF_RANGE:
        throw std::out_of_range(message);
    case UHA_DOMAIN_ERROR:
        throw std::domain_error(message);
    case UHA_LOGIC_ERROR:
        throw std::logic_error(message);
    default:
        throw std::runtime_error(message);
    }
}

// Runs engine draws on the caller's std::mt19937_64: the engine state is
// handed to the library and taken back, so the caller's engine advances
// exactly as if the draws had used it directly.
class EngineBridge {
public:
    explicit EngineBridge(std::mt19937_64& engine) : engine_(engine)
    {
        check(uha_rng_create(0, &rng_));
        std::ostringstream os;
        os << engine_;
        check(uha_rng_set_state(rng_, os.str().c_str()));
    }
    EngineBridge(const EngineBridge&) = delete;
    EngineBridge& operator=(const EngineBridge&) = delete;
    ~EngineBridge() { uha_rng_destroy(rng_); }

    uha_rng* get() const noexcept { return rng_; }

    // Copies the advanced state back into the caller's engine.
    void commit()
    {
        uint64_t length = 0;
        check(uha_rng_state(rng_, nullptr, 0, &length));
        std::string text(length, '\0');
        check(uha_rng_state(rng_, text.data(), length, &length));
        std::istringstream is(text);
        is >> engine_;
    }

private:
    std::mt19937_64& engine_;
    uha_rng* rng_ = nullptr;
};

// Owns one engine index handle.
struct IndexHandle {
    uha_index* index = nullptr;
    IndexHandle() = default;
    explicit IndexHandle(uha_index* i) : index(i) {}
    IndexHandle(const IndexHandle&) = delete;
    IndexHandle& operator=(const IndexHandle&) = delete;
    ~IndexHandle() { uha_index_destroy(index); }
};

// Owns one engine workspace handle.
struct WorkspaceHandle {
    uha_workspace* workspace = nullptr;
    WorkspaceHandle() = default;
    explicit WorkspaceHandle(uha_workspace* w) : workspace(w) {}
    WorkspaceHandle(const WorkspaceHandle&) = delete;
    WorkspaceHandle& operator=(const WorkspaceHandle&) = delete;
    ~WorkspaceHandle() { uha_workspace_destroy(workspace); }
};

inline std::string device_name_of(const uha_index* index)
{
    char name[256] = {};
    check(uha_index_device(index, nullptr, name, sizeof(name)));
    return name;
}

inline int device_of(const uha_index* index)
{
    int device = 0;
    check(uha_index_device(index, &device, nullptr, 0));
    return device;
}

}  // namespace ultrahigh_ann::engine
