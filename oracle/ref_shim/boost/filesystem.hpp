// Empty stand-in: the reference's math translation unit includes this header but uses none of it.
#pragma once
