// World deltas of the brick-world service: block edits reported by the game
// (aero_lbm_simulation_submit_world_deltas) patch the host copy of a brick's
// static fields — obstacle, fan footprints, heat plumes, open faces — with the
// reference's rules (native/src/aero_lbm_simulation_bridge.cpp:1885-2825);
// the device copy follows at the brick's next device use.
#include <algorithm>
#include <cmath>
#include <unordered_set>

#include "brick_world.h"

namespace aero {
namespace bw {

namespace {

constexpr int kFanLength = 5;        // k_client_fan_force_length_cells (simulation_bridge.cpp:507)
constexpr int kFanRadius = 1;        // k_client_fan_force_radius_cells (:508)
constexpr int kPlumeHeight = 4;      // k_client_heat_plume_height_cells (:509)
constexpr float kHeatCoupling = 0.85f;  // k_client_heat_coupling_to_adjacent_air (:510)
// Java face order of open_face_mask bits: -y, +y, -z, +z, -x, +x (:492-496)
constexpr int kJavaFace[6][3] = {{0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}, {-1, 0, 0}, {1, 0, 0}};
// fan direction codes 1..6: -x, +x, -y, +y, -z, +z (:497-505)
constexpr int kFanDir[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};

int fan_axis(int dir) { return dir <= 2 ? 0 : (dir <= 4 ? 1 : 2); }
uint8_t fan_kind(int dir) { return (dir >= 1 && dir <= 6) ? (uint8_t)(31 + dir) : 0u; }
int cell_index(int n, int x, int y, int z) { return (x * n + y) * n + z; }

// offset (a, b) across the fan axis
void lane(int axis, int a, int b, int& x, int& y, int& z) {
    if (axis == 0) {
        y += a;
        z += b;
    } else if (axis == 1) {
        x += a;
        z += b;
    } else {
        x += a;
        y += b;
    }
}

// ---- whole-brick derivation from the source fields (:1885-2098)
bool local_solid(const StaticFields& s, int n, int x, int y, int z) {
    if (x < 0 || y < 0 || z < 0 || x >= n || y >= n || z >= n) return true;
    const size_t c = (size_t)cell_index(n, x, y, z);
    return c >= s.obstacle.size() || s.obstacle[c] != 0;
}

uint16_t local_open_faces(const StaticFields& s, int n, int x, int y, int z) {
    if (local_solid(s, n, x, y, z)) return 0u;
    uint16_t m = 0;
    for (int f = 0; f < 6; ++f)
        if (!local_solid(s, n, x + kJavaFace[f][0], y + kJavaFace[f][1], z + kJavaFace[f][2])) m = (uint16_t)(m | (1u << f));
    return m;
}

// Brick-local view of a world patch: cells outside the brick count as solid
// and hold no sources; the patched cell takes its new values.
struct PatchView {
    const StaticFields& s;
    Coord brick;
    int n;
    const AeroLbmWorldDelta& d;
    bool new_solid;
    uint8_t new_fan;
    float new_power;

    bool local(int wx, int wy, int wz, int& lx, int& ly, int& lz) const {
        lx = wx - brick.x * n;
        ly = wy - brick.y * n;
        lz = wz - brick.z * n;
        return lx >= 0 && ly >= 0 && lz >= 0 && lx < n && ly < n && lz < n;
    }
    bool is_source(int wx, int wy, int wz) const { return wx == d.x && wy == d.y && wz == d.z; }
    bool solid(int wx, int wy, int wz) const {
        if (is_source(wx, wy, wz)) return new_solid;
        int lx, ly, lz;
        if (!local(wx, wy, wz, lx, ly, lz)) return true;
        const size_t c = (size_t)cell_index(n, lx, ly, lz);
        return c >= s.obstacle.size() || s.obstacle[c] != 0;
    }
    uint8_t fan_dir(int wx, int wy, int wz) const {
        if (is_source(wx, wy, wz)) return new_fan;
        int lx, ly, lz;
        if (!local(wx, wy, wz, lx, ly, lz)) return 0u;
        const size_t c = (size_t)cell_index(n, lx, ly, lz);
        return c < s.source_fan_dir.size() ? s.source_fan_dir[c] : 0u;
    }
    float power(int wx, int wy, int wz) const {
        if (is_source(wx, wy, wz)) return new_power;
        int lx, ly, lz;
        if (!local(wx, wy, wz, lx, ly, lz)) return 0.0f;
        const size_t c = (size_t)cell_index(n, lx, ly, lz);
        return c < s.source_emitter_power.size() ? s.source_emitter_power[c] : 0.0f;
    }
    // fan_path_clear_for_world_cell (:2244-2285)
    bool fan_clear(int fx, int fy, int fz, int dir, int distance, int a, int b) const {
        int x = fx, y = fy, z = fz;
        lane(fan_axis(dir), a, b, x, y, z);
        for (int step = 1; step < distance; ++step)
            if (solid(x + kFanDir[dir][0] * step, y + kFanDir[dir][1] * step, z + kFanDir[dir][2] * step)) return false;
        return true;
    }
    // compute_source_surface_kind_for_cell (:2287-2343)
    uint8_t surface_kind(int lx, int ly, int lz) const {
        const int wx = brick.x * n + lx, wy = brick.y * n + ly, wz = brick.z * n + lz;
        if (solid(wx, wy, wz)) return 0u;
        for (int dir = 1; dir <= 6; ++dir) {
            const int axis = fan_axis(dir);
            for (int dist = 1; dist <= kFanLength; ++dist) {
                const int ax = wx - kFanDir[dir][0] * dist, ay = wy - kFanDir[dir][1] * dist, az = wz - kFanDir[dir][2] * dist;
                for (int a = -kFanRadius; a <= kFanRadius; ++a)
                    for (int b = -kFanRadius; b <= kFanRadius; ++b) {
                        int fx = ax, fy = ay, fz = az;
                        lane(axis, -a, -b, fx, fy, fz);
                        if (fan_dir(fx, fy, fz) != dir) continue;
                        if (!fan_clear(fx, fy, fz, dir, dist, a, b)) continue;
                        return fan_kind(dir);
                    }
            }
        }
        return 0u;
    }
    // compute_source_open_face_mask_for_cell (:2345-2375)
    uint16_t open_faces(int lx, int ly, int lz) const {
        const int wx = brick.x * n + lx, wy = brick.y * n + ly, wz = brick.z * n + lz;
        if (solid(wx, wy, wz)) return 0u;
        uint16_t m = 0;
        for (int f = 0; f < 6; ++f)
            if (!solid(wx + kJavaFace[f][0], wy + kJavaFace[f][1], wz + kJavaFace[f][2])) m = (uint16_t)(m | (1u << f));
        return m;
    }
    // heat_path_clear_for_world_cell (:2377-2393)
    bool heat_clear(int x, int sy, int z, int ty) const {
        for (int y = sy + 1; y < ty; ++y)
            if (solid(x, y, z)) return false;
        return true;
    }
    // compute_source_emitter_power_for_cell (:2395-2445)
    float emitter_power(int lx, int ly, int lz) const {
        const int wx = brick.x * n + lx, wy = brick.y * n + ly, wz = brick.z * n + lz;
        if (solid(wx, wy, wz)) return 0.0f;
        const float direct = power(wx, wy, wz);
        if (direct > 0.0f) return direct;
        float coupled = 0.0f;
        for (int dist = 1; dist <= kPlumeHeight; ++dist) {
            const int sy = wy - dist;
            const float below = power(wx, sy, wz);
            if (below <= 0.0f || !heat_clear(wx, sy, wz, wy)) continue;
            coupled += below * kHeatCoupling / (float)(dist * dist);
        }
        return coupled;
    }
};

void add_cell(const Coord& brick, int n, std::unordered_set<int>& out, int wx, int wy, int wz) {
    const int lx = wx - brick.x * n, ly = wy - brick.y * n, lz = wz - brick.z * n;
    if (lx >= 0 && ly >= 0 && lz >= 0 && lx < n && ly < n && lz < n) out.insert(cell_index(n, lx, ly, lz));
}

void add_fan_disk(const Coord& brick, int n, std::unordered_set<int>& out, int cx, int cy, int cz, int dir) {
    const int axis = fan_axis(dir);
    for (int a = -kFanRadius; a <= kFanRadius; ++a)
        for (int b = -kFanRadius; b <= kFanRadius; ++b) {
            int x = cx, y = cy, z = cz;
            lane(axis, a, b, x, y, z);
            add_cell(brick, n, out, x, y, z);
        }
}

void add_fan_footprint(const Coord& brick, int n, std::unordered_set<int>& out, int sx, int sy, int sz, int dir) {
    if (dir <= 0 || dir > 6) return;
    for (int dist = 1; dist <= kFanLength; ++dist)
        add_fan_disk(brick, n, out, sx + kFanDir[dir][0] * dist, sy + kFanDir[dir][1] * dist, sz + kFanDir[dir][2] * dist, dir);
}

// add_source_delta_affected_cells (:2171-2225)
void affected_cells(const Coord& brick, int n, std::unordered_set<int>& out, const AeroLbmWorldDelta& d, uint8_t old_fan,
                    uint8_t new_fan, bool obstacle_changed, bool heat_changed) {
    add_cell(brick, n, out, d.x, d.y, d.z);
    for (const auto& o : kJavaFace) add_cell(brick, n, out, d.x + o[0], d.y + o[1], d.z + o[2]);
    if (old_fan != 0) add_fan_footprint(brick, n, out, d.x, d.y, d.z, old_fan);
    if (new_fan != 0) add_fan_footprint(brick, n, out, d.x, d.y, d.z, new_fan);
    if (obstacle_changed) {
        for (int dir = 1; dir <= 6; ++dir)
            for (int dist = 1; dist <= kFanLength; ++dist)
                add_fan_disk(brick, n, out, d.x + kFanDir[dir][0] * dist, d.y + kFanDir[dir][1] * dist,
                             d.z + kFanDir[dir][2] * dist, dir);
        for (int dist = 1; dist <= kPlumeHeight; ++dist) add_cell(brick, n, out, d.x, d.y + dist, d.z);
    }
    if (heat_changed)
        for (int dist = 0; dist <= kPlumeHeight; ++dist) add_cell(brick, n, out, d.x, d.y + dist, d.z);
}

// apply_source_delta_to_brick (:2481-2658)
void apply_source_delta(World& w, const Coord& coord, Brick& brick, const AeroLbmWorldDelta& d) {
    const int n = w.brick_size;
    if (!brick.stat || brick.stat->obstacle.size() != (size_t)n * n * n) return;
    const bool old_solid = (d.data1 & 0x1) != 0, new_solid = (d.data1 & 0x2) != 0;
    const uint8_t old_fan = (uint8_t)((d.data1 >> 8) & 0xFF), new_fan = (uint8_t)((d.data1 >> 16) & 0xFF);
    const float old_power = std::isfinite(d.value0) ? d.value0 : 0.0f;
    const float new_power = std::isfinite(d.value1) ? d.value1 : 0.0f;
    std::unordered_set<int> cells;
    affected_cells(coord, n, cells, d, old_fan, new_fan, old_solid != new_solid, old_power != new_power);
    const int slx = d.x - coord.x * n, sly = d.y - coord.y * n, slz = d.z - coord.z * n;
    const bool source_here = slx >= 0 && sly >= 0 && slz >= 0 && slx < n && sly < n && slz < n;
    if (cells.empty() && !source_here) return;
    StaticFields& s = *brick.stat;
    ensure_source_fields(s, (size_t)n * n * n);
    if (source_here) {
        const int c = cell_index(n, slx, sly, slz);
        s.obstacle[c] = new_solid ? 1u : 0u;
        s.source_fan_dir[c] = std::min<uint8_t>(new_fan, 6u);
        s.source_emitter_power[c] = new_power;
        cells.insert(c);
    }
    const PatchView v{s, coord, n, d, new_solid, new_fan, new_power};
    bool changed = false;
    for (int c : cells) {
        if (c < 0 || (size_t)c >= s.obstacle.size()) continue;
        const int lx = c / (n * n), ly = (c / n) % n, lz = c % n;
        const uint8_t ob = v.solid(coord.x * n + lx, coord.y * n + ly, coord.z * n + lz) ? 1u : 0u;
        const uint8_t kind = v.surface_kind(lx, ly, lz);
        const uint16_t faces = v.open_faces(lx, ly, lz);
        const float power = v.emitter_power(lx, ly, lz);
        const bool cell_changed = s.obstacle[c] != ob || s.surface_kind[c] != kind || s.open_face_mask[c] != faces ||
                                  s.emitter_power[c] != power;
        s.obstacle[c] = ob;
        s.surface_kind[c] = kind;
        s.open_face_mask[c] = faces;
        s.emitter_power[c] = power;
        if ((size_t)c * 6 + 6 <= s.face_sky.size()) std::fill_n(s.face_sky.begin() + (std::ptrdiff_t)c * 6, 6, 0u);
        if ((size_t)c * 6 + 6 <= s.face_direct.size()) std::fill_n(s.face_direct.begin() + (std::ptrdiff_t)c * 6, 6, 0u);
        if (cell_changed) {
            brick.pending_patch_cells.push_back(c);
            changed = true;
        }
    }
    // the host copy changed in any case; the dynamic state takes the
    // constraints only when a constraint field changed
    static_changed(w, brick, changed);
    if (changed) {
        brick.forcing_dirty = true;
        brick.geometry_dirty = brick.pending_reinit = false;
        brick.active = true;
        brick.last_active_epoch = w.epoch;
    }
}

int floor_div(int v, int d) {
    if (d <= 0) return 0;
    const int q = v / d, r = v % d;
    return (r != 0 && v < 0) ? q - 1 : q;
}

}  // namespace

void ensure_source_fields(StaticFields& s, size_t cells) {
    if (s.source_fan_dir.size() != cells) s.source_fan_dir.assign(cells, 0u);
    if (s.source_emitter_power.size() != cells) s.source_emitter_power.assign(cells, 0.0f);
}

// rebuild_static_region_derived_fields_from_sources (simulation_bridge.cpp:1987-2096)
void rebuild_static_from_sources(StaticFields& s, int n) {
    const size_t cells = (size_t)n * n * n;
    if (n <= 0 || s.obstacle.size() != cells) return;
    s.surface_kind.assign(cells, 0u);
    if (s.open_face_mask.size() != cells) s.open_face_mask.assign(cells, 0u);
    s.emitter_power.assign(cells, 0.0f);
    ensure_source_fields(s, cells);
    for (int x = 0; x < n; ++x)
        for (int y = 0; y < n; ++y)
            for (int z = 0; z < n; ++z) s.open_face_mask[cell_index(n, x, y, z)] = local_open_faces(s, n, x, y, z);
    for (int fx = 0; fx < n; ++fx)
        for (int fy = 0; fy < n; ++fy)
            for (int fz = 0; fz < n; ++fz) {
                const int dir = std::min<uint8_t>(s.source_fan_dir[cell_index(n, fx, fy, fz)], 6u);
                if (dir == 0) continue;
                const int axis = fan_axis(dir);
                for (int dist = 1; dist <= kFanLength; ++dist) {
                    const int cx = fx + kFanDir[dir][0] * dist, cy = fy + kFanDir[dir][1] * dist, cz = fz + kFanDir[dir][2] * dist;
                    for (int a = -kFanRadius; a <= kFanRadius; ++a)
                        for (int b = -kFanRadius; b <= kFanRadius; ++b) {
                            int tx = cx, ty = cy, tz = cz;
                            lane(axis, a, b, tx, ty, tz);
                            if (local_solid(s, n, tx, ty, tz)) continue;
                            // the lane from the fan to this cell must be open (local_fan_path_clear, :1935-1966)
                            int lx = fx, ly = fy, lz = fz;
                            lane(axis, a, b, lx, ly, lz);
                            bool clear = true;
                            for (int step = 1; step < dist && clear; ++step)
                                clear = !local_solid(s, n, lx + kFanDir[dir][0] * step, ly + kFanDir[dir][1] * step,
                                                     lz + kFanDir[dir][2] * step);
                            if (!clear) continue;
                            s.surface_kind[cell_index(n, tx, ty, tz)] = fan_kind(dir);
                        }
                }
            }
    for (int sx = 0; sx < n; ++sx)
        for (int sy = 0; sy < n; ++sy)
            for (int sz = 0; sz < n; ++sz) {
                const float p = s.source_emitter_power[cell_index(n, sx, sy, sz)];
                if (!(p > 0.0f) || !std::isfinite(p)) continue;
                for (int dist = 0; dist <= kPlumeHeight; ++dist) {
                    const int ty = sy + dist;
                    if (ty < 0 || ty >= n || local_solid(s, n, sx, ty, sz)) continue;
                    bool clear = true;
                    for (int y = sy + 1; y < ty && clear; ++y) clear = !local_solid(s, n, sx, y, sz);
                    if (!clear) continue;
                    s.emitter_power[cell_index(n, sx, ty, sz)] += dist == 0 ? p : p * kHeatCoupling / (float)(dist * dist);
                }
            }
}

// apply_brick_world_delta (simulation_bridge.cpp:2687-2771)
void apply_world_delta(World& w, const AeroLbmWorldDelta& d) {
    const int n = w.brick_size;
    const Coord coord{floor_div(d.x, n), floor_div(d.y, n), floor_div(d.z, n)};
    switch (d.type) {
        case 10:  // k_world_delta_brick_static_source_patch
            for (auto& [c, b] : w.bricks) apply_source_delta(w, c, b, d);
            break;
        case 8: {  // k_world_delta_brick_static_cell_patch
            auto it = w.bricks.find(coord);
            if (it == w.bricks.end()) break;
            Brick& b = it->second;
            if (!b.stat || b.stat->obstacle.size() != (size_t)n * n * n) break;
            const int lx = d.x - coord.x * n, ly = d.y - coord.y * n, lz = d.z - coord.z * n;
            if (lx < 0 || ly < 0 || lz < 0 || lx >= n || ly >= n || lz >= n) break;
            const int c = cell_index(n, lx, ly, lz);
            StaticFields& s = *b.stat;
            const uint8_t ob = (d.data1 & 0x1) != 0 ? 1u : 0u;
            const uint8_t kind = (uint8_t)((d.data1 >> 8) & 0xFF);
            const uint16_t faces = (uint16_t)(d.data2 & 0xFF);
            const float power = std::isfinite(d.value0) ? d.value0 : 0.0f;
            const bool cell_changed = s.obstacle[c] != ob || s.surface_kind[c] != kind || s.open_face_mask[c] != faces ||
                                      s.emitter_power[c] != power;
            s.obstacle[c] = ob;
            s.surface_kind[c] = kind;
            s.open_face_mask[c] = faces;
            s.emitter_power[c] = power;
            std::fill_n(s.face_sky.begin() + (std::ptrdiff_t)c * 6, 6, 0u);
            std::fill_n(s.face_direct.begin() + (std::ptrdiff_t)c * 6, 6, 0u);
            static_changed(w, b, true);
            b.forcing_dirty = b.forcing_dirty || cell_changed;
            if (cell_changed) b.pending_patch_cells.push_back(c);
            b.active = true;
            b.last_active_epoch = w.epoch;
            break;
        }
        case 1:
            mark_brick(w, coord, true, false, false);
            break;
        case 2:
        case 3:
            // mark_brick_and_neighbor_reinit (simulation_bridge.cpp:1849-1863)
            mark_brick(w, coord, true, false, true);
            for (const auto& o : {Coord{-1, 0, 0}, Coord{1, 0, 0}, Coord{0, -1, 0}, Coord{0, 1, 0}, Coord{0, 0, -1}, Coord{0, 0, 1}}) {
                const Coord nc{coord.x + o.x, coord.y + o.y, coord.z + o.z};
                if (w.bricks.count(nc)) mark_brick(w, nc, false, false, true);
            }
            break;
        case 4:
        case 5:
            mark_brick(w, coord, false, true, false);
            break;
        default:
            break;
    }
}

}  // namespace bw
}  // namespace aero
