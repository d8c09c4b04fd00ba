#pragma once
#include_next <dirent.h>
#include "windows.h"
