// Stand-in for the kiwi logging header (pkg kiwi v0.3.1, not vendored in the reference).
#pragma once
namespace kiwi {
namespace logs {
template <class... A> inline void v(A&&...) {}
template <class... A> inline void d(A&&...) {}
template <class... A> inline void i(A&&...) {}
template <class... A> inline void w(A&&...) {}
template <class... A> inline void e(A&&...) {}
template <class... A> inline void s(A&&...) {}
}  // namespace logs
}  // namespace kiwi
