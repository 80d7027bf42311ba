// Host stand-in for nlohmann::json (oracle/_ref build only). The reference's math and
// optimizer headers declare json constructors and serialisers that the hot-path kernels never
// call; this minimal value type lets those declarations compile. It holds numbers and nested
// lists, nothing more.
#pragma once

#include <initializer_list>
#include <string>
#include <utility>
#include <vector>

namespace nlohmann {

class json {
public:
    json() = default;
    json(double v) : num_(v) {}
    json(float v) : num_(v) {}
    json(int v) : num_(v) {}
    json(unsigned int v) : num_(v) {}
    json(const char*) {}
    json(const std::string&) {}
    json(std::initializer_list<json> items) : items_(items) {}
    template <typename T>
    json(const std::pair<std::string, T>&) {}

    json& operator[](int i) {
        if (items_.size() <= (size_t)i) items_.resize((size_t)i + 1);
        return items_[(size_t)i];
    }
    const json& operator[](int i) const { return items_.at((size_t)i); }
    json& operator[](const char*) { return *this; }
    const json& operator[](const char*) const { return *this; }
    bool contains(const char*) const { return false; }
    operator double() const { return num_; }
    operator float() const { return (float)num_; }
    operator unsigned int() const { return (unsigned int)num_; }

private:
    double num_ = 0.0;
    std::vector<json> items_;
};

}  // namespace nlohmann
