// Stand-in for the header-only Boost.Any, which is not installed here.
// The reference uses boost::any only to carry parameter maps; std::any has
// the same interface for those uses and carries no arithmetic.
#pragma once
#include <any>
namespace boost { using std::any; using std::any_cast; using bad_any_cast = std::bad_any_cast; }
