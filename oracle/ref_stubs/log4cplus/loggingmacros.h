#pragma once
#include "logger.h"
#define LOG4CPLUS_TRACE(logger, message) do {} while (0)
#define LOG4CPLUS_DEBUG(logger, message) do {} while (0)
#define LOG4CPLUS_INFO(logger, message) do {} while (0)
#define LOG4CPLUS_WARN(logger, message) do {} while (0)
#define LOG4CPLUS_ERROR(logger, message) do {} while (0)
#define LOG4CPLUS_FATAL(logger, message) do {} while (0)
