// Minimal stand-in for log4cplus: loggers exist as members but never log on this path.
#pragma once
namespace log4cplus {
class Logger {
public:
    static Logger getInstance(const char *) { return Logger(); }
};
}
#ifndef LOG4CPLUS_TEXT
#define LOG4CPLUS_TEXT(text) text
#endif
