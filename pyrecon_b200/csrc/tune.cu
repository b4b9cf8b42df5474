// Run-time tuning table: named integer knobs, each keyed by an integer (a mesh axis length), that the
// kernel launchers read when they launch.  The autotuner (pyrecon_b200/tuning.py) times the variants a
// knob selects on the device at hand and stores its choices here; unset entries fall back to the
// launcher's built-in default.  A change bumps a generation counter that the captured multigrid
// graphs include in their keys, so a graph never replays kernels chosen under older settings.
#include "common.cuh"

#include <map>
#include <stdlib.h>
#include <mutex>
#include <string>
#include <utility>

namespace prc {

namespace {
std::mutex g_tune_mutex;
std::map<std::pair<std::string, int>, int> g_tune;
unsigned g_tune_generation = 0;
}  // namespace

int tune_get(const char* name, int key, int dflt) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune.find(std::make_pair(std::string(name), key));
    return it == g_tune.end() ? dflt : it->second;
}

unsigned tune_generation() {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    return g_tune_generation;
}

bool pdl_enabled() {
    static const bool on = [] {
        const char* v = getenv("PRC_PDL");
        return !(v != nullptr && v[0] == '0');
    }();
    return on;
}

}  // namespace prc

extern "C" {

PRC_API int prc_tune_set(const char* name, int key, int value) {
    if (!name || !name[0]) return PRC_ERR_ARG;
    std::lock_guard<std::mutex> lock(prc::g_tune_mutex);
    const auto k = std::make_pair(std::string(name), key);
    if (value < 0) prc::g_tune.erase(k);
    else prc::g_tune[k] = value;
    prc::g_tune_generation++;
    return PRC_OK;
}

PRC_API int prc_tune_get(const char* name, int key, int dflt) {
    if (!name) return dflt;
    return prc::tune_get(name, key, dflt);
}

PRC_API void prc_tune_clear(void) {
    std::lock_guard<std::mutex> lock(prc::g_tune_mutex);
    prc::g_tune.clear();
    prc::g_tune_generation++;
}

}  // extern "C"
