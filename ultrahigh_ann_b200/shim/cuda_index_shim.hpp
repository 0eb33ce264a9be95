// Shared state of the shimmed index classes: an engine index handle, its
// workspaces, and the reference's argument checks in the reference's order.
#pragma once

#include "ultrahigh_ann/core/index_space_usage.hpp"

#include "shim_support.hpp"

#include <cstdint>
#include <limits>
#include <span>
#include <stdexcept>
#include <string>

namespace ultrahigh_ann::engine {

struct IndexState {
    IndexHandle handle;
    std::size_t dimension = 0;  // original query dimension
    int device = 0;
    std::string device_name;

    void attach(uha_index* index, std::size_t d)
    {
        handle.index = index;
        dimension = d;
        device = device_of(index);
        device_name = device_name_of(index);
    }
    IndexSpaceUsage usage() const noexcept
    {
        uha_space_usage u{};
        if (uha_index_space_usage(handle.index, &u) != UHA_OK) {
            return IndexSpaceUsage{};
        }
        return IndexSpaceUsage{u.index_payload_bytes, u.query_workspace_payload_bytes,
                               u.unique_query_coordinates, u.sampled_multiplicity};
    }
};

struct WorkspaceState {
    WorkspaceHandle handle;
    const void* owner = nullptr;
    std::size_t maximum_batch_size = 0;
    std::size_t payload_bytes = 0;

    void attach(const IndexState& index, const void* owner_key, std::size_t batch)
    {
        check(uha_workspace_create(index.handle.index, batch, &handle.workspace));
        owner = owner_key;
        uint64_t b = 0;
        uint64_t p = 0;
        check(uha_workspace_info(handle.workspace, &b, &p));
        maximum_batch_size = b;
        payload_bytes = p;
    }
};

// Argument checks of the reference facades, then the engine query. When
// `check_dimension_first` the query-dimension check precedes the output-size
// check (hierarchical facades); otherwise it follows it (sampled facades).
inline void facade_query(const IndexState& index, WorkspaceState* ws,
                         const void* owner, std::span<const float> queries,
                         std::size_t query_count, std::span<std::size_t> output,
                         uha_strategy strategy, const std::string& name,
                         bool check_dimension_first)
{
    if (ws == nullptr || ws->owner != owner) {
        throw std::invalid_argument("CUDA " + name +
                                    " workspace belongs to a different index");
    }
    if (query_count > ws->maximum_batch_size) {
        throw std::invalid_argument("query count exceeds CUDA " + name +
                                    " workspace capacity");
    }
    auto check_dimension = [&] {
        if (index.dimension != 0 &&
            query_count > std::numeric_limits<std::size_t>::max() / index.dimension) {
            throw std::length_error("CUDA " + name + " query batch size overflows");
        }
        if (queries.size() != query_count * index.dimension) {
            throw std::invalid_argument(
                "query batch dimensions do not match original dimension");
        }
    };
    if (check_dimension_first) {
        check_dimension();
    }
    if (output.size() != query_count) {
        throw std::invalid_argument("CUDA " + name +
                                    " output size does not match query count");
    }
    if (query_count == 0) {
        return;
    }
    if (!check_dimension_first) {
        check_dimension();
    }
    check(uha_query(index.handle.index, ws->handle.workspace, queries.data(),
                    query_count, 0, strategy,
                    reinterpret_cast<std::uint64_t*>(output.data()), nullptr));
}

}  // namespace ultrahigh_ann::engine
