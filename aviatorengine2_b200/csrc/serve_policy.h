// serve_policy.h - host-side decisions of the serving loop, kept free of CUDA
// so they can be exercised on any machine:
//
//   * Arena: first-fit placement of request images inside one device block
//     that is allocated once, so admitting a request never calls cudaMalloc;
//   * Policy: admission in arrival order by memory footprint and resident
//     slots, and the ordering of instance moves against the requests of a
//     scene (a request renders the scene as it was when it was submitted).
//     Each scene has `frame_sets` copies of its per-frame arrays.  A version
//     is materialized (refit, then written into a free copy) when a queued
//     request needs it, or eagerly as the newest state when a copy is free;
//     moves that no request will see are coalesced into the next one (moves
//     carry absolute transforms).  A copy is free when no outstanding request
//     renders the version it holds.
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
    uint32_t copy = 0;     // set at admission: the copy holding its version
};

class Policy {
  public:
    void configure(uint64_t arena_bytes, uint32_t max_resident, uint32_t frame_sets = 2);
    // A new scene; its version 0 lives in copy 0.
    uint32_t add_scene();
    uint32_t scenes() const { return uint32_t(newest_.size()); }
    // Queues a request; fills in its scene version.  False when it can never
    // fit (footprint above the whole arena) or the scene is unknown.
    bool submit(PolicyRequest &r);
    // Queues an instance move of `scene`; returns the version it creates
    // (0 for an unknown scene).  Requests submitted after it see it.
    uint32_t move(uint32_t scene);
    // The next move to apply: its scene, the version to materialize (the
    // oldest version a queued request needs, else the newest submitted; the
    // versions below it that no request needs are coalesced) and the copy
    // to write it into.  False when nothing is to be applied or no copy of
    // the scene is free.
    bool next_move(uint32_t &scene, uint32_t &version, uint32_t &copy) const;
    void move_applied(uint32_t scene, uint32_t version, uint32_t copy);
    // The next request to admit (arrival order; requests whose version is
    // not materialized yet are passed over, a request that does not fit stops
    // the scan so large requests are not starved).  Places it in the arena
    // and names the copy it renders from.
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
    uint32_t newest(uint32_t scene) const { return newest_[scene]; }
    uint32_t submitted(uint32_t scene) const { return submitted_moves_[scene]; }
    uint32_t frame_sets() const { return frame_sets_; }
    // The copy holding `version` of `scene`, or -1.
    int copy_of(uint32_t scene, uint32_t version) const;

  private:
    uint32_t outstanding(uint32_t scene, int64_t version) const;
    Arena arena_;
    uint32_t max_resident_ = 1, resident_ = 0, frame_sets_ = 2;
    std::deque<PolicyRequest> pending_;
    std::map<uint64_t, std::pair<PolicyRequest, uint64_t>> active_;  // id -> (request, offset)
    std::vector<uint32_t> newest_, submitted_moves_;
    std::vector<std::vector<int64_t>> copy_version_;                  // per scene, per copy; -1 = empty
    std::map<std::pair<uint32_t, uint32_t>, uint32_t> outstanding_;  // (scene, version) -> pending + active
};

}  // namespace ae
