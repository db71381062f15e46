#pragma once
#include "logger.h"
