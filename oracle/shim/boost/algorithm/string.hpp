// Small stand-in for the handful of Boost.StringAlgo calls the reference makes while
// parsing tag names and component paths (split / is_any_of / trim_*_if / starts_with /
// contains / find_last). Written for building the reference as the test oracle only;
// the semantics follow the Boost documentation for std::string arguments.
#pragma once

#include <algorithm>
#include <string>
#include <vector>

namespace boost
{
namespace algorithm
{

struct any_of_pred
{
  std::string set;
  bool operator()(char c) const
  {
    return set.find(c) != std::string::npos;
  }
};

inline any_of_pred is_any_of(const std::string &chars)
{
  return any_of_pred{chars};
}

// Tokens between separators; adjacent separators give empty tokens (Boost's default
// token_compress_off behaviour).
template <typename Seq, typename Pred>
Seq &split(Seq &out, const std::string &input, Pred pred)
{
  out.clear();
  std::string cur;
  for (char c : input)
  {
    if (pred(c))
    {
      out.push_back(cur);
      cur.clear();
    }
    else
    {
      cur.push_back(c);
    }
  }
  out.push_back(cur);
  return out;
}

template <typename Pred>
void trim_left_if(std::string &s, Pred pred)
{
  std::size_t i = 0;
  while (i < s.size() && pred(s[i]))
    ++i;
  s.erase(0, i);
}

template <typename Pred>
void trim_right_if(std::string &s, Pred pred)
{
  std::size_t n = s.size();
  while (n > 0 && pred(s[n - 1]))
    --n;
  s.erase(n);
}

inline bool starts_with(const std::string &s, const std::string &prefix)
{
  return s.size() >= prefix.size() && s.compare(0, prefix.size(), prefix) == 0;
}

inline bool contains(const std::string &s, const std::string &what)
{
  return s.find(what) != std::string::npos;
}

// Iterator range of the last occurrence of 'what' in 's' (empty range at s.end() when absent).
struct string_range
{
  std::string::iterator b, e;
  std::string::iterator begin() const
  {
    return b;
  }
  std::string::iterator end() const
  {
    return e;
  }
};

inline string_range find_last(std::string &s, const std::string &what)
{
  const std::size_t pos = s.rfind(what);
  if (pos == std::string::npos || what.empty())
    return string_range{s.end(), s.end()};
  return string_range{s.begin() + pos, s.begin() + pos + what.size()};
}

} // namespace algorithm

using algorithm::contains;
using algorithm::is_any_of;
using algorithm::split;
using algorithm::starts_with;

} // namespace boost
