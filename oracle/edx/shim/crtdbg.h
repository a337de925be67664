// empty: the MSVC debug runtime header that EDXUtil/Core/Types.h includes
#pragma once
