// Generated by gen_crmath_tables.py (80-digit decimal arithmetic). Do not edit.
// Each table is a brace initializer; crmath.cuh instantiates a host and a device copy.
#pragma once

// log(n / 128), n = 85 .. 171
#define CMPMC_CR_LOGC { \
    {-0x1.a33440224fa79p-2, 0x1.ba8062860ae23p-57}, \
    {-0x1.973a3431356aep-2, 0x1.89d2816cf838fp-57}, \
    {-0x1.8b639a88b2df5p-2, 0x1.70f2f38238303p-56}, \
    {-0x1.7fafa3bd8151cp-2, 0x1.219024acd3b77p-58}, \
    {-0x1.741d876c67bb1p-2, -0x1.84a4ee3059583p-56}, \
    {-0x1.68ac83e9c6a14p-2, -0x1.a64eadd740178p-58}, \
    {-0x1.5d5bddf595f30p-2, 0x1.6541148cbb8a2p-56}, \
    {-0x1.522ae0738a3d8p-2, 0x1.8f7e9b38a6979p-57}, \
    {-0x1.4718dc271c41bp-2, -0x1.8fb4c14c56eefp-60}, \
    {-0x1.3c25277333184p-2, 0x1.2ad27e50a8ec6p-56}, \
    {-0x1.314f1e1d35ce4p-2, 0x1.3d69909e5c3dcp-56}, \
    {-0x1.269621134db92p-2, -0x1.e0efadd9db02bp-56}, \
    {-0x1.1bf99635a6b95p-2, 0x1.12aeb84249223p-57}, \
    {-0x1.1178e8227e47cp-2, 0x1.0e63a5f01c691p-57}, \
    {-0x1.07138604d5862p-2, -0x1.cdb16ed4e9138p-56}, \
    {-0x1.f991c6cb3b379p-3, -0x1.f665066f980a2p-57}, \
    {-0x1.e530effe71012p-3, -0x1.2276041f43042p-59}, \
    {-0x1.d1037f2655e7bp-3, -0x1.60629242471a2p-57}, \
    {-0x1.bd087383bd8adp-3, -0x1.dd355f6a516d7p-60}, \
    {-0x1.a93ed3c8ad9e3p-3, -0x1.bcafa9de97203p-57}, \
    {-0x1.95a5adcf7017fp-3, -0x1.142c507fb7a3dp-58}, \
    {-0x1.823c16551a3c2p-3, 0x1.1232ce70be781p-57}, \
    {-0x1.6f0128b756abcp-3, 0x1.8de59c21e166cp-57}, \
    {-0x1.5bf406b543db2p-3, 0x1.1f5b44c0df7e7p-61}, \
    {-0x1.4913d8333b561p-3, 0x1.0d5604930f135p-58}, \
    {-0x1.365fcb0159016p-3, -0x1.7d411a5b944adp-58}, \
    {-0x1.23d712a49c202p-3, 0x1.6e38161051d69p-57}, \
    {-0x1.1178e8227e47cp-3, 0x1.0e63a5f01c691p-58}, \
    {-0x1.fe89139dbd566p-4, 0x1.ac9f4215f9393p-58}, \
    {-0x1.da727638446a2p-4, -0x1.401fa71733019p-58}, \
    {-0x1.b6ac88dad5b1cp-4, 0x1.0057eed1ca59fp-59}, \
    {-0x1.9335e5d594989p-4, 0x1.478a85704ccb7p-58}, \
    {-0x1.700d30aeac0e1p-4, 0x1.72566212cdd05p-61}, \
    {-0x1.4d3115d207eacp-4, -0x1.769f42c7842ccp-58}, \
    {-0x1.2aa04a44717a5p-4, 0x1.d15d38d2fa3f7p-58}, \
    {-0x1.08598b59e3a07p-4, 0x1.dd7009902bf32p-58}, \
    {-0x1.ccb73cdddb2ccp-5, 0x1.e48fb0500efd4p-59}, \
    {-0x1.894aa149fb343p-5, -0x1.a8be97660a23dp-60}, \
    {-0x1.466aed42de3eap-5, 0x1.cdd6f7f4a137ep-59}, \
    {-0x1.0415d89e74444p-5, -0x1.c05cf1d753622p-59}, \
    {-0x1.8492528c8cabfp-6, 0x1.d192d0619fa67p-60}, \
    {-0x1.0205658935847p-6, -0x1.27c8e8416e71fp-60}, \
    {-0x1.010157588de71p-7, -0x1.46662d417ced0p-62}, \
    {0x0.0p+0, 0x0.0p+0}, \
    {0x1.fe02a6b106789p-8, -0x1.e44b7e3711ebfp-67}, \
    {0x1.fc0a8b0fc03e4p-7, -0x1.83092c59642a1p-62}, \
    {0x1.7b91b07d5b11bp-6, -0x1.5b602ace3a510p-60}, \
    {0x1.f829b0e783300p-6, 0x1.33e3f04f1ef23p-60}, \
    {0x1.39e87b9febd60p-5, -0x1.5bfa937f551bbp-59}, \
    {0x1.77458f632dcfcp-5, 0x1.18d3ca87b9296p-59}, \
    {0x1.b42dd711971bfp-5, -0x1.eb9759c130499p-60}, \
    {0x1.f0a30c01162a6p-5, 0x1.85f325c5bbacdp-59}, \
    {0x1.16536eea37ae1p-4, -0x1.79da3e8c22cdap-60}, \
    {0x1.341d7961bd1d1p-4, -0x1.b599f227becbbp-58}, \
    {0x1.51b073f06183fp-4, 0x1.a49e39a1a8be4p-58}, \
    {0x1.6f0d28ae56b4cp-4, -0x1.906d99184b992p-58}, \
    {0x1.8c345d6319b21p-4, -0x1.4a697ab3424a9p-61}, \
    {0x1.a926d3a4ad563p-4, 0x1.942f48aa70ea9p-58}, \
    {0x1.c5e548f5bc743p-4, 0x1.5d617ef8161b1p-60}, \
    {0x1.e27076e2af2e6p-4, -0x1.61578001e0162p-60}, \
    {0x1.fec9131dbeabbp-4, -0x1.5746b9981b36cp-58}, \
    {0x1.0d77e7cd08e59p-3, 0x1.9a5dc5e9030acp-57}, \
    {0x1.1b72ad52f67a0p-3, 0x1.483023472cd74p-58}, \
    {0x1.29552f81ff523p-3, 0x1.301771c407dbfp-57}, \
    {0x1.371fc201e8f74p-3, 0x1.de6cb62af18a0p-58}, \
    {0x1.44d2b6ccb7d1ep-3, 0x1.9f4f6543e1f88p-57}, \
    {0x1.526e5e3a1b438p-3, -0x1.746ff8a470d3ap-57}, \
    {0x1.5ff3070a793d4p-3, -0x1.bc60efafc6f6ep-58}, \
    {0x1.6d60fe719d21dp-3, -0x1.caae268ecd179p-57}, \
    {0x1.7ab890210d909p-3, 0x1.be36b2d6a0608p-59}, \
    {0x1.87fa06520c911p-3, -0x1.bf7fdbfa08d9ap-57}, \
    {0x1.9525a9cf456b4p-3, 0x1.d904c1d4e2e26p-57}, \
    {0x1.a23bc1fe2b563p-3, 0x1.93711b07a998cp-59}, \
    {0x1.af3c94e80bff3p-3, -0x1.398cff3641985p-58}, \
    {0x1.bc286742d8cd6p-3, 0x1.4fce744870f55p-58}, \
    {0x1.c8ff7c79a9a22p-3, -0x1.4f689f8434012p-57}, \
    {0x1.d5c216b4fbb91p-3, 0x1.6e443597e4d40p-57}, \
    {0x1.e27076e2af2e6p-3, -0x1.61578001e0162p-59}, \
    {0x1.ef0adcbdc5936p-3, 0x1.48637950dc20dp-57}, \
    {0x1.fb9186d5e3e2bp-3, -0x1.caaae64f21acbp-57}, \
    {0x1.0402594b4d041p-2, -0x1.28ec217a5022dp-57}, \
    {0x1.0a324e27390e3p-2, 0x1.7dcfde8061c03p-56}, \
    {0x1.1058bf9ae4ad5p-2, 0x1.89fa0ab4cb31dp-58}, \
    {0x1.1675cababa60ep-2, 0x1.ce63eab883717p-61}, \
    {0x1.1c898c16999fbp-2, -0x1.0e5c62aff1c44p-60}, \
    {0x1.22941fbcf7966p-2, -0x1.76f5eb09628afp-56}, \
    {0x1.2895a13de86a3p-2, 0x1.7ad24c13f040ep-56}, \
  }
#define CMPMC_CR_LN2_HI 0x1.62e42fefa39efp-1
#define CMPMC_CR_LN2_LO 0x1.abc9e3b39803fp-56
#define CMPMC_CR_LN2_H42 0x1.62e42fefa3800p-1
#define CMPMC_CR_LN2_T42 0x1.ef35793c76730p-45
#define CMPMC_CR_INV6_HI 0x1.5555555555555p-3
#define CMPMC_CR_INV6_LO 0x1.5555555555555p-57
#define CMPMC_CR_INV24_HI 0x1.5555555555555p-5
#define CMPMC_CR_INV24_LO 0x1.5555555555555p-59
// 1 / (2k + 1)
#define CMPMC_CR_INVODD { \
    {0x1.0000000000000p+0, 0x0.0p+0}, \
    {0x1.5555555555555p-2, 0x1.5555555555555p-56}, \
    {0x1.999999999999ap-3, -0x1.999999999999ap-57}, \
    {0x1.2492492492492p-3, 0x1.2492492492492p-57}, \
    {0x1.c71c71c71c71cp-4, 0x1.c71c71c71c71cp-58}, \
    {0x1.745d1745d1746p-4, -0x1.745d1745d1746p-59}, \
    {0x1.3b13b13b13b14p-4, -0x1.3b13b13b13b14p-58}, \
    {0x1.1111111111111p-4, 0x1.1111111111111p-60}, \
    {0x1.e1e1e1e1e1e1ep-5, 0x1.e1e1e1e1e1e1ep-61}, \
    {0x1.af286bca1af28p-5, 0x1.af286bca1af28p-59}, \
    {0x1.8618618618618p-5, 0x1.8618618618618p-59}, \
    {0x1.642c8590b2164p-5, 0x1.642c8590b2164p-60}, \
  }
// (-1)^k / (2k + 1)!
#define CMPMC_CR_SINC { \
    {0x1.0000000000000p+0, 0x0.0p+0}, \
    {-0x1.5555555555555p-3, -0x1.5555555555555p-57}, \
    {0x1.1111111111111p-7, 0x1.1111111111111p-63}, \
    {-0x1.a01a01a01a01ap-13, -0x1.a01a01a01a01ap-73}, \
    {0x1.71de3a556c734p-19, -0x1.c154f8ddc6c00p-73}, \
    {-0x1.ae64567f544e4p-26, 0x1.c062e06d1f209p-80}, \
    {0x1.6124613a86d09p-33, 0x1.f28e0cc748ebep-87}, \
    {-0x1.ae7f3e733b81fp-41, -0x1.1d8656b0ee8cbp-97}, \
    {0x1.952c77030ad4ap-49, 0x1.ac981465ddc6cp-103}, \
    {-0x1.2f49b46814157p-57, -0x1.2650f61dbdcb4p-112}, \
    {0x1.71b8ef6dcf572p-66, -0x1.d043ae40c4647p-120}, \
    {-0x1.761b41316381ap-75, 0x1.3423c7d91404fp-130}, \
    {0x1.3f3ccdd165fa9p-84, -0x1.58ddadf344487p-139}, \
    {-0x1.d1ab1c2dccea3p-94, -0x1.054d0c78aea14p-149}, \
    {0x1.259f98b4358adp-103, 0x1.eaf8c39dd9bc5p-157}, \
    {-0x1.434d2e783f5bcp-113, -0x1.0b87b91be9affp-167}, \
  }
// (-1)^k / (2k)!
#define CMPMC_CR_COSC { \
    {0x1.0000000000000p+0, 0x0.0p+0}, \
    {-0x1.0000000000000p-1, 0x0.0p+0}, \
    {0x1.5555555555555p-5, 0x1.5555555555555p-59}, \
    {-0x1.6c16c16c16c17p-10, 0x1.f49f49f49f49fp-65}, \
    {0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-76}, \
    {-0x1.27e4fb7789f5cp-22, -0x1.cbbc05b4fa99ap-76}, \
    {0x1.1eed8eff8d898p-29, -0x1.2aec959e14c06p-83}, \
    {-0x1.93974a8c07c9dp-37, -0x1.05d6f8a2efd1fp-92}, \
    {0x1.ae7f3e733b81fp-45, 0x1.1d8656b0ee8cbp-101}, \
    {-0x1.6827863b97d97p-53, -0x1.eec01221a8b0bp-107}, \
    {0x1.e542ba4020225p-62, 0x1.ea72b4afe3c2fp-120}, \
    {-0x1.0ce396db7f853p-70, 0x1.aebcdbd20331cp-124}, \
    {0x1.f2cf01972f578p-80, -0x1.9ada5fcc1ab14p-135}, \
    {-0x1.88e85fc6a4e5ap-89, 0x1.71c37ebd16540p-143}, \
    {0x1.0a18a2635085dp-98, 0x1.b9e2e28e1aa54p-153}, \
    {-0x1.3932c5047d60ep-108, -0x1.832b7b530a627p-162}, \
    {0x1.434d2e783f5bcp-118, 0x1.0b87b91be9affp-172}, \
  }
// pi/2 = kPio2[0] + kPio2[1] + kPio2[2] + kPio2[3]; the first two carry 33 bits
#define CMPMC_CR_PIO2_1 0x1.921fb54400000p+0
#define CMPMC_CR_PIO2_2 0x1.0b4611a600000p-34
#define CMPMC_CR_PIO2_3 0x1.3198a2e037073p-69
#define CMPMC_CR_PIO2_4 0x1.129024e088a68p-123
#define CMPMC_CR_TWO_OVER_PI 0x1.45f306dc9c883p-1

