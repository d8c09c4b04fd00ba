#pragma once
#include_next <dirent.h>
#include "windows.h"
// some of the reference's Win32 dirent.h copies also name the entry type Dirent
typedef struct dirent Dirent;
