/*
 * Declarations that let the reference's include/config.h compile in the
 * checker build (TEST INFRASTRUCTURE ONLY).  toml++ is absent here and the
 * checker never parses TOML: parse_file throws, and every lookup yields an
 * empty view.  The checker calls the reference's MBIR drivers with a
 * ReconParams whose fields it sets directly.
 */
#ifndef ORACLE_SHIM_TOML_H
#define ORACLE_SHIM_TOML_H

#include <cstddef>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>

namespace toml {

class table;
class array;

class node {
  public:
    const table *as_table() const { return nullptr; }
    const array *as_array() const { return nullptr; }
    template <class T>
    std::optional<T> value() const { return std::nullopt; }
    template <class T>
    T value_or(T d) const { return d; }
};

class node_view {
  public:
    explicit operator bool() const { return false; }
    node_view operator[](std::string_view) const { return {}; }
    const table *as_table() const { return nullptr; }
    const array *as_array() const { return nullptr; }
    template <class T>
    std::optional<T> value() const { return std::nullopt; }
    template <class T>
    T value_or(T d) const { return d; }
};

class array {
  public:
    const node *begin() const { return nullptr; }
    const node *end() const { return nullptr; }
    size_t size() const { return 0; }
    const node &operator[](size_t) const { throw std::out_of_range("toml stub: empty array"); }
};

class table {
  public:
    node_view operator[](std::string_view) const { return {}; }
    bool contains(std::string_view) const { return false; }
};

class parse_error : public std::runtime_error {
  public:
    using std::runtime_error::runtime_error;
    std::string_view description() const noexcept { return what(); }
};

inline table parse_file(std::string_view) { throw parse_error("toml++ is not available in the checker build"); }

}  // namespace toml

#endif
