// utils/read_config.cpp -- Config (behaviour of src/utils/read_config.cpp:18-64).
#include <cctype>
#include <fstream>
#include <iostream>
#include <sstream>
#include <stdexcept>

#include "utils.hpp"

namespace Gaukuk {

Config& Config::getInstance() {
    static Config instance;
    return instance;
}

void Config::loadFromFile(const std::string& filename) {
    std::ifstream file(filename);
    if (!file) throw std::invalid_argument("Could not open the input file");
    std::string line;
    while (std::getline(file, line)) {
        line = trim(line);
        if (line.empty() || line[0] == '#') continue;
        const size_t pos = line.find('=');
        if (pos != std::string::npos) line[pos] = ' ';
        std::istringstream iss(line);
        std::string key;
        Real value;
        if (iss >> key >> value) {
            data[key] = value;
        } else {
            std::cout << key << std::endl;
            std::cerr << "Warning: Invalid line in config file: " << line << std::endl;
        }
    }
}

Real Config::get(const std::string& key, Real defaultValue) {
    auto it = data.find(key);
    return it == data.end() ? defaultValue : it->second;
}

std::string Config::trim(const std::string& str) {
    size_t b = 0, e = str.size();
    while (b < e && std::isspace(static_cast<unsigned char>(str[b]))) ++b;
    while (e > b && std::isspace(static_cast<unsigned char>(str[e - 1]))) --e;
    return str.substr(b, e - b);
}

}  // namespace Gaukuk
