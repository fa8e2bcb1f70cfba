// Minimal stand-in for spdlog 1.15 used only to compile the reference's
// sources into the test oracle (oracle/_ref).  The reference's release build
// compiles its SPDLOG_DEBUG calls out (SPDLOG_ACTIVE_LEVEL=WARN); this shim
// drops every log macro.
#pragma once
#define SPDLOG_DEBUG(...) ((void)0)
#define SPDLOG_ERROR(...) ((void)0)
#define SPDLOG_INFO(...) ((void)0)
#define SPDLOG_WARN(...) ((void)0)
#define SPDLOG_TRACE(...) ((void)0)
