#include "generator.h"

#include "maboss_b200_mirror.h"
#include "timer.h"

generator::generator(driver& drv) : drv_(drv) {}

std::string generator::generate_code() const
{
	timer_stats t("generator> generate_code");
	mb_model m = drv_.model();
	size_t len = 0;
	mirror::check(mb_model_generate_code(m, nullptr, 0, &len), "generate_code");
	std::string code(len + 1, '\0');
	mirror::check(mb_model_generate_code(m, code.data(), code.size(), &len), "generate_code");
	code.resize(len);
	return code;
}
