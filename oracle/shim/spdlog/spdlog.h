// Test-only stand-in for the logging library the reference headers include; every call is a no-op.
#pragma once
namespace spdlog { template<typename... A> void error(A &&...) {} template<typename... A> void warn(A &&...) {} template<typename... A> void info(A &&...) {} template<typename... A> void debug(A &&...) {} }
