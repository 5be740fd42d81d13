// utils/utils.hpp -- the run-time configuration of the host interface.
//
// Config is the reference's singleton (src/utils/utils.hpp:12-22,
// read_config.cpp): key = value lines, every value a Real, a missing key
// reads as the default passed to get (0 when none).
#pragma once

#include <map>
#include <string>

#include "../gaukuk.hpp"

namespace Gaukuk {

class Config {
public:
    static Config& getInstance();
    void loadFromFile(const std::string& filename);
    Real get(const std::string& key, Real defaultValue = 0.0);
    bool has(const std::string& key) const { return data.count(key) != 0; }
    void set(const std::string& key, Real value) { data[key] = value; }

private:
    Config() = default;
    std::map<std::string, Real> data;
    static std::string trim(const std::string& str);
};

namespace GMath {
inline Real SQR(Real a) { return a * a; }
}  // namespace GMath

}  // namespace Gaukuk
