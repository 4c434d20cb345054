// Logger.h -- logging of the ktt:: surface (internal).
//
// Levels and behaviour of KTT 2.1.0 Source/Utility/Logger/Logger.cpp:10-80: messages at or below the
// configured level (Off < Error < Warning < Info < Debug; default Info) are written with a
// "[Level] KTT: " prefix to the configured stream (std::clog by default) or file.
#pragma once

#include <fstream>
#include <iostream>
#include <memory>
#include <mutex>
#include <string>

#include <ktt/KttTypes.h>

namespace ktt::log
{

struct State
{
    LoggingLevel level = LoggingLevel::Info;
    std::ostream* stream = &std::clog;
    std::unique_ptr<std::ofstream> file;
    std::mutex mutex;
};

inline State& state()
{
    static State s;
    return s;
}

inline void write(const LoggingLevel level, const char* tag, const std::string& message)
{
    State& s = state();

    if (static_cast<int>(level) > static_cast<int>(s.level) || s.level == LoggingLevel::Off)
    {
        return;
    }

    std::lock_guard<std::mutex> lock(s.mutex);
    *s.stream << "[" << tag << "] KTT: " << message << std::endl;
}

inline void Error(const std::string& m) { write(LoggingLevel::Error, "Error", m); }
inline void Warning(const std::string& m) { write(LoggingLevel::Warning, "Warning", m); }
inline void Info(const std::string& m) { write(LoggingLevel::Info, "Info", m); }
inline void Debug(const std::string& m) { write(LoggingLevel::Debug, "Debug", m); }

} // namespace ktt::log
