// serve_policy.h - host-side decisions of the serving loop, kept free of CUDA
// so they can be exercised on any machine:
//
//   * Arena: first-fit placement of request images inside one device block
//     that is allocated once, so admitting a request never calls cudaMalloc;
//   * Policy: admission in arrival order by memory footprint and resident
//     slots, and the ordering of instance moves against the requests of a
//     scene (a request renders the scene as it was when it was submitted).
//     Each scene has `frame_sets` copies of its per-frame arrays; version v
//     lives in copy v % frame_sets, so a move to version v + 1 may be applied
//     once no request of version v + 1 - frame_sets is outstanding, while
//     requests of the newer versions still run.
#pragma once
#include <cstdint>
#include <deque>
#include <map>
#include <utility>
#include <vector>

namespace ae {

class Arena {
  public:
    static constexpr uint64_t kAlign = 256;
    static constexpr uint64_t kNone = ~0ull;
    explicit Arena(uint64_t bytes = 0) { reset(bytes); }
    void reset(uint64_t bytes);
    // Offset of a new block of at least `bytes` (rounded up to kAlign), or
    // kNone when no free range is large enough.
    uint64_t alloc(uint64_t bytes);
    // Returns a block to the free list, merging it with free neighbours.
    bool release(uint64_t offset);
    uint64_t capacity() const { return cap_; }
    uint64_t used() const { return used_; }
    uint64_t largest_free() const;
    size_t free_ranges() const { return free_.size(); }

  private:
    uint64_t cap_ = 0, used_ = 0;
    std::map<uint64_t, uint64_t> free_;  // offset -> size
    std::map<uint64_t, uint64_t> live_;  // offset -> size
};

inline uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

struct PolicyRequest {
    uint64_t id = 0;
    uint32_t scene = 0;
    uint64_t footprint = 0;
    uint32_t version = 0;  // moves of its scene submitted before it
};

class Policy {
  public:
    void configure(uint64_t arena_bytes, uint32_t max_resident, uint32_t frame_sets = 2);
    uint32_t add_scene();
    uint32_t scenes() const { return uint32_t(applied_.size()); }
    // Queues a request; fills in its scene version.  False when it can never
    // fit (footprint above the whole arena) or the scene is unknown.
    bool submit(PolicyRequest &r);
    // Queues an instance move of `scene`; requests submitted after it see it.
    bool move(uint32_t scene);
    // A scene whose oldest queued move may be applied now: every request of
    // the version whose copy the move overwrites has completed.
    bool next_move(uint32_t &scene) const;
    void move_applied(uint32_t scene);
    // The next request to admit (arrival order; requests waiting for a move
    // of their scene are passed over, a request that does not fit stops the
    // scan so large requests are not starved).  Places it in the arena.
    bool next_admission(PolicyRequest &out, uint64_t &offset);
    // Releases a completed request's arena block and resident slot.
    void completed(uint64_t id);
    // Removes a request still queued (not admitted); false when it is not
    // queued.  An admitted request is withdrawn through completed() once its
    // work in flight has drained.
    bool withdraw(uint64_t id);
    // Drops every queued request (server shutdown); returns their ids.
    std::vector<uint64_t> cancel_pending();

    uint32_t resident() const { return resident_; }
    size_t pending() const { return pending_.size(); }
    const Arena &arena() const { return arena_; }
    uint32_t applied(uint32_t scene) const { return applied_[scene]; }

  private:
    Arena arena_;
    uint32_t max_resident_ = 1, resident_ = 0, frame_sets_ = 2;
    std::deque<PolicyRequest> pending_;
    std::map<uint64_t, std::pair<PolicyRequest, uint64_t>> active_;  // id -> (request, offset)
    std::vector<uint32_t> applied_, submitted_moves_;
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> outstanding_;  // (scene, version) -> pending + active
};

}  // namespace ae
