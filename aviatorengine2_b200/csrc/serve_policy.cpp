// serve_policy.cpp - arena placement and admission order of the serving loop,
// plus ae_serve_policy_simulate, which drives the same Policy through a
// synthetic event list on the host (no GPU) so its invariants can be tested.
#include "serve_policy.h"

#include <algorithm>

#include "../../include/ae_b200.h"

namespace ae {

void Arena::reset(uint64_t bytes) {
    cap_ = bytes / kAlign * kAlign;
    used_ = 0;
    free_.clear();
    live_.clear();
    if (cap_) free_[0] = cap_;
}

uint64_t Arena::alloc(uint64_t bytes) {
    const uint64_t need = align_up(std::max<uint64_t>(bytes, 1), kAlign);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
        if (it->second < need) continue;
        const uint64_t off = it->first, size = it->second;
        free_.erase(it);
        if (size > need) free_[off + need] = size - need;
        live_[off] = need;
        used_ += need;
        return off;
    }
    return kNone;
}

bool Arena::release(uint64_t offset) {
    auto lv = live_.find(offset);
    if (lv == live_.end()) return false;
    uint64_t off = offset, size = lv->second;
    live_.erase(lv);
    used_ -= size;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + size == next->first) {
        size += next->second;
        next = free_.erase(next);
    }
    if (next != free_.begin()) {
        auto prev = std::prev(next);
        if (prev->first + prev->second == off) {
            off = prev->first;
            size += prev->second;
            free_.erase(prev);
        }
    }
    free_[off] = size;
    return true;
}

uint64_t Arena::largest_free() const {
    uint64_t m = 0;
    for (const auto &f : free_) m = std::max(m, f.second);
    return m;
}

void Policy::configure(uint64_t arena_bytes, uint32_t max_resident, uint32_t frame_sets) {
    arena_.reset(arena_bytes);
    max_resident_ = std::max(max_resident, 1u);
    frame_sets_ = std::max(frame_sets, 1u);
}

uint32_t Policy::add_scene() {
    newest_.push_back(0);
    submitted_moves_.push_back(0);
    std::vector<int64_t> copies(frame_sets_, -1);
    copies[0] = 0;
    copy_version_.push_back(copies);
    return uint32_t(newest_.size() - 1);
}

bool Policy::submit(PolicyRequest &r) {
    if (r.scene >= newest_.size()) return false;
    if (align_up(r.footprint, Arena::kAlign) > arena_.capacity()) return false;
    r.version = submitted_moves_[r.scene];
    pending_.push_back(r);
    outstanding_[{r.scene, r.version}]++;
    return true;
}

uint32_t Policy::move(uint32_t scene) {
    if (scene >= newest_.size()) return 0;
    return ++submitted_moves_[scene];
}

uint32_t Policy::outstanding(uint32_t scene, int64_t version) const {
    if (version < 0) return 0;
    auto it = outstanding_.find({scene, uint32_t(version)});
    return it == outstanding_.end() ? 0 : it->second;
}

int Policy::copy_of(uint32_t scene, uint32_t version) const {
    const std::vector<int64_t> &cv = copy_version_[scene];
    for (uint32_t c = 0; c < cv.size(); c++)
        if (cv[c] == int64_t(version)) return int(c);
    return -1;
}

bool Policy::next_move(uint32_t &scene, uint32_t &version, uint32_t &copy) const {
    for (uint32_t s = 0; s < newest_.size(); s++) {
        if (submitted_moves_[s] == newest_[s]) continue;
        // The oldest version above the newest that a queued request renders;
        // with none, the newest submitted state.
        uint32_t target = submitted_moves_[s];
        for (auto it = outstanding_.lower_bound({s, newest_[s] + 1}); it != outstanding_.end() && it->first.first == s;
             ++it) {
            if (it->second) {
                target = it->first.second;
                break;
            }
        }
        const std::vector<int64_t> &cv = copy_version_[s];
        for (uint32_t c = 0; c < cv.size(); c++) {
            if (cv[c] < 0 || outstanding(s, cv[c]) == 0) {
                scene = s;
                version = target;
                copy = c;
                return true;
            }
        }
    }
    return false;
}

void Policy::move_applied(uint32_t scene, uint32_t version, uint32_t copy) {
    const int64_t old = copy_version_[scene][copy];
    if (old >= 0) outstanding_.erase({scene, uint32_t(old)});
    copy_version_[scene][copy] = version;
    newest_[scene] = version;
}

bool Policy::next_admission(PolicyRequest &out, uint64_t &offset) {
    if (resident_ >= max_resident_) return false;
    for (auto it = pending_.begin(); it != pending_.end(); ++it) {
        // A request waits until its version is materialized; that copy stays
        // intact until every request of the version is done.
        const int copy = copy_of(it->scene, it->version);
        if (copy < 0) continue;
        const uint64_t off = arena_.alloc(it->footprint);
        if (off == Arena::kNone) return false;  // arrival order: later requests wait too
        out = *it;
        out.copy = uint32_t(copy);
        offset = off;
        pending_.erase(it);
        active_[out.id] = {out, off};
        resident_++;
        return true;
    }
    return false;
}

void Policy::completed(uint64_t id) {
    auto it = active_.find(id);
    if (it == active_.end()) return;
    const PolicyRequest &r = it->second.first;
    arena_.release(it->second.second);
    auto o = outstanding_.find({r.scene, r.version});
    if (o != outstanding_.end() && o->second) o->second--;
    resident_--;
    active_.erase(it);
}

bool Policy::withdraw(uint64_t id) {
    for (auto it = pending_.begin(); it != pending_.end(); ++it) {
        if (it->id != id) continue;
        auto o = outstanding_.find({it->scene, it->version});
        if (o != outstanding_.end() && o->second) o->second--;
        pending_.erase(it);
        return true;
    }
    return false;
}

std::vector<uint64_t> Policy::cancel_pending() {
    std::vector<uint64_t> ids;
    for (const PolicyRequest &r : pending_) {
        ids.push_back(r.id);
        auto o = outstanding_.find({r.scene, r.version});
        if (o != outstanding_.end() && o->second) o->second--;
    }
    pending_.clear();
    return ids;
}

}  // namespace ae

using namespace ae;

// Discrete-time run of the admission policy: events arrive at their tick (in
// list order within a tick); each tick applies every move that may apply
// (coalescing the ones no request needs), admits what fits, then advances
// admitted requests by one tick of service.
extern "C" int ae_serve_policy_simulate(const ae_policy_event *events, uint32_t n, uint64_t arena_bytes,
                                        uint32_t max_resident, uint32_t n_scenes, uint32_t frame_sets,
                                        uint32_t max_ticks, ae_policy_outcome *out) {
    if ((n && (!events || !out)) || n_scenes == 0 || frame_sets == 0) return AE_ERR_INVALID;
    Policy P;
    P.configure(arena_bytes, max_resident, frame_sets);
    for (uint32_t s = 0; s < n_scenes; s++) P.add_scene();
    for (uint32_t i = 0; i < n; i++) {
        out[i].admit_tick = out[i].done_tick = -1;
        out[i].version = 0;
        out[i].status = AE_OK;
        out[i].offset = ~0ull;
        if (events[i].scene >= n_scenes || (i && events[i].tick < events[i - 1].tick)) return AE_ERR_INVALID;
    }
    std::vector<std::deque<uint32_t>> moves(n_scenes);  // event index of each queued move
    std::map<uint64_t, uint32_t> remaining;             // admitted request -> service ticks left
    uint32_t next_event = 0, finished = 0, expected = 0;
    for (uint32_t i = 0; i < n; i++) expected += 1;
    for (int64_t t = 0; t <= int64_t(max_ticks) && finished < expected; t++) {
        while (next_event < n && events[next_event].tick <= t) {
            const ae_policy_event &e = events[next_event];
            if (e.kind == AE_POLICY_MOVE) {
                out[next_event].version = P.move(e.scene);
                moves[e.scene].push_back(next_event);
            } else if (e.kind == AE_POLICY_CANCEL) {
                // Withdraw request event `footprint`: a queued one at once, an
                // admitted one as if its work in flight drained this tick.  A
                // request that has not arrived yet or has finished is left as is.
                const uint64_t target = e.footprint;
                out[next_event].admit_tick = out[next_event].done_tick = int32_t(t);
                finished++;
                if (target < n && events[target].kind == AE_POLICY_REQUEST && out[target].done_tick < 0 &&
                    out[target].status == AE_OK) {
                    if (P.withdraw(target)) {
                        out[target].status = AE_ERR_CANCELLED;
                        out[target].done_tick = int32_t(t);
                        finished++;
                    } else if (remaining.count(target)) {
                        remaining.erase(target);
                        P.completed(target);
                        out[target].status = AE_ERR_CANCELLED;
                        out[target].done_tick = int32_t(t);
                        finished++;
                    }
                }
            } else {
                PolicyRequest r;
                r.id = next_event;
                r.scene = e.scene;
                r.footprint = e.footprint;
                if (!P.submit(r)) {
                    out[next_event].status = AE_ERR_REJECTED;
                    finished++;
                } else {
                    out[next_event].version = r.version;
                }
            }
            next_event++;
        }
        bool progress = true;
        while (progress) {
            progress = false;
            uint32_t s, v, c;
            while (P.next_move(s, v, c)) {
                // Moves below the materialized version are coalesced into it.
                while (!moves[s].empty()) {
                    const uint32_t mi = moves[s].front();
                    if (out[mi].version > v) break;
                    moves[s].pop_front();
                    out[mi].admit_tick = out[mi].done_tick = int32_t(t);
                    out[mi].offset = out[mi].version == v ? uint64_t(c) : ~0ull;
                    finished++;
                }
                P.move_applied(s, v, c);
                progress = true;
            }
            PolicyRequest r;
            uint64_t off;
            while (P.next_admission(r, off)) {
                out[r.id].admit_tick = int32_t(t);
                out[r.id].offset = off;
                remaining[r.id] = std::max(events[r.id].service_ticks, 1u);
                progress = true;
            }
        }
        for (auto it = remaining.begin(); it != remaining.end();) {
            if (--it->second == 0) {
                out[it->first].done_tick = int32_t(t);
                P.completed(it->first);
                finished++;
                it = remaining.erase(it);
            } else {
                ++it;
            }
        }
    }
    return finished == expected ? AE_OK : AE_ERR_TIMEOUT;
}
